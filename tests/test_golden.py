"""Golden fixtures written from the reference build (tests/golden/make_golden.py):
the CPU oracle must reproduce them bit for bit, the device path to 1e-12
relative (bit for bit in practice).  The fixtures need no reference tree."""
import copy
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from make_golden import CASES  # noqa: E402

from arcos_b200 import workloads  # noqa: E402
from parity_util import max_ulp, port_tree, rel_err  # noqa: E402


def load(name):
    (kind, kw), steps, flavour = CASES[name]
    pb = getattr(workloads, kind)(**kw)
    if name == "theta_ref_exact":
        pb.params.per_plane = False
    gold = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    for g in range(len(pb.specs)):
        for s in range(pb.model.no_species):
            assert np.array_equal(gold[f"in_g{g}_s{s}"], pb.dens[g][s]), "workload generator changed"
    return pb, gold, steps, flavour


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_golden(name):
    pb, gold, steps, flavour = load(name)
    E = pb.family_E[0] if pb.family_E else None
    port = port_tree(pb, zero_all=(flavour == "zero_all"),
                     per_plane=(flavour == "per_plane" or (pb.specs[0].ntheta == 1)) if name.startswith("theta") else None,
                     E=E)
    dts = [port.rk2(50.0)[0] for _ in range(steps)]
    assert np.array_equal(np.array(dts), gold["dts"])
    for g in range(len(pb.specs)):
        for s in range(pb.model.no_species):
            assert max_ulp(port.dens(g, s), gold[f"out_g{g}_s{s}"]) == 0, (name, g, s)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_device_matches_golden(cuda_device, name):
    from arcos_b200.cdr import CdrTree
    pb, gold, steps, flavour = load(name)
    if name.startswith("theta"):
        pb.params.per_plane = flavour == "per_plane"
    dev = CdrTree(pb.params, pb.model, pb.specs, exact=True)
    for g, per in enumerate(pb.dens):
        for s, a in enumerate(per):
            dev.upload(g, "dens", a, s)
    for f, E in enumerate(pb.family_E):
        dev.set_family_field(f, *E)
    dev.set_fixed_field(pb.fields)
    if len(pb.specs) == 1:
        dts = dev.run(steps, 50.0)[0]
    else:
        dts = [dev.cdr_rk2(50.0) for _ in range(steps)]
    assert np.array_equal(np.array(dts), gold["dts"])
    for g in range(len(pb.specs)):
        for s in range(pb.model.no_species):
            a = dev.download(g, "dens", s)
            b = gold[f"out_g{g}_s{s}"]
            assert rel_err(a, b) <= 1e-12, (name, g, s, rel_err(a, b))
            assert max_ulp(a, b) == 0, (name, g, s, max_ulp(a, b))
