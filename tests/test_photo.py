"""Photoionization (photo_calc, src/photo.c:313-345, the entry that ends the
reactions list, src/rt.c:38-47 and reaction.c:203-210): the impact
ionization counter d_dens[dummyplus] / ntheta is the source of one
Helmholtz problem per photo term (es = the term's lambda, per theta mode
lambda = -w2k[m]), whose solution times A is added to d_dens of electrons
and of the photo ions.

CPU part (this file): the oracle (oracle/cdr_port.c port_photo_calc) against
the reference's own photo.c, compiled from the reference sources with the
Helmholtz stand-in of oracle/poisson_host.c in place of FISHPACK, bit for
bit, on 2-D and 3-D grids, with the field fixed or solved in the loop.
The device side is in test_gpu_photo.py.
"""
import copy

import numpy as np
import pytest

from arcos_b200 import workloads
from oracle import bind
from parity_util import max_ulp, port_tree

needs_ref = pytest.mark.skipif(not bind.ref_available(), reason="reference build absent")


def ref_tree(pb, field_mode):
    t = bind.RefTree(copy.deepcopy(pb.params), pb.model, pb.specs, field_mode=field_mode)
    for g, per in enumerate(pb.dens):
        for s, a in enumerate(per):
            t.dens(g, s)[...] = a
    if field_mode == bind.FIELD_FIXED:
        for g, (er, ez, et) in enumerate(pb.fields):
            t.set_fixed_field(g, er, ez, et if et is not None else pb.specs[g].zeros())
    return t


@needs_ref
@pytest.mark.parametrize("ntheta,field_mode,field", [
    (1, bind.FIELD_FIXED, "uniform"), (1, bind.FIELD_FIXED, "wavy"), (1, bind.FIELD_POISSON, "uniform"),
    (4, bind.FIELD_FIXED, "uniform"), (4, bind.FIELD_POISSON, "uniform"), (5, bind.FIELD_POISSON, "uniform")])
def test_port_photo_matches_reference(ntheta, field_mode, field):
    pb = workloads.photo(nr=20, nz=36, ntheta=ntheta, noise=0.3, seed=3, field=field)
    port = port_tree(pb, field_mode=field_mode, per_plane=True)
    ref = ref_tree(pb, field_mode)
    if field_mode == bind.FIELD_POISSON:
        port.call("port_calc_charge")
        ref.call("ref_calc_charge_r")
    for _ in range(3):
        h_ref = ref.rk2_sw(50.0, per_plane=True, zero_all=False) if ntheta > 1 else ref.rk2(50.0)
        assert port.rk2(50.0)[0] == h_ref
    for w in ("dens", "d_dens"):
        for s in range(pb.model.no_species):
            assert max_ulp(port.array(0, w, s), ref.array(0, w, s)) == 0, (w, s)
    # the photo ions come from photoionization alone, and they are there
    assert np.max(port.dens(0, 4)) > 0


def test_photo_terms_add_linearly():
    """The photo contribution is linear in the terms' weights: doubling both
    A doubles d_dens of the photo ions (a host check of the oracle's
    photo_calc, on the first derivative)."""
    res = []
    for scale in (1.0, 2.0):
        pb = workloads.photo(nr=16, nz=24, noise=0.2, seed=1,
                             terms=((0.02 * scale, -0.8), (0.05 * scale, -6.0)))
        port = port_tree(pb)
        port.rk2(50.0)
        res.append(port.array(0, "d_dens", 4).copy())
    a, b = res
    assert np.max(np.abs(b - 2 * a)) <= 1e-12 * np.max(np.abs(b))
