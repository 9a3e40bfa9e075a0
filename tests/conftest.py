"""Test configuration: the ``gpu`` marker, and the oracle libraries built on
demand (the reference build only where the reference sources exist)."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    port = os.path.join(ROOT, "oracle", "liboracle_port.so")
    if not os.path.exists(port):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "port"], check=True)
    ref = os.path.join(ROOT, "oracle", "_ref", "libarcos_ref.so")
    if not os.path.exists(ref):
        # oracle/Makefile knows where the reference sources are; without them
        # (a machine that only has the prebuilt files) the build is skipped
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=False,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda_device():
    if not gpu_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    return 0
