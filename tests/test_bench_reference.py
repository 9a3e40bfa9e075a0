"""The bench's reference arm (CPU only): one JSON line with the contract's
keys, the reference's serial step on every host core, and nothing from the
ranks other than 0."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                           "--steps", "1", "--warmup", "1"], cwd=ROOT, env=env,
                          capture_output=True, text=True, timeout=900)


def test_reference_arm_line():
    p = _run({"RANK": "0"})
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [x for x in p.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1 and p.stdout.strip() == lines[0]
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    cores = len(os.sched_getaffinity(0))
    assert d["cpu_baseline"]["cores"] == max(1, min(cores, 64))
    assert d["cpu_baseline"]["kind"] in ("reference", "port")
    assert "the whole grid" in d["cpu_baseline"]["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    p = _run({"RANK": "1"})
    assert p.returncode == 0 and p.stdout.strip() == ""
