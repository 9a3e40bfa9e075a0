"""The drop-in claims at link level: the reference's own C, linked against
the device library, against the reference as built for the oracle.

* Seam route (oracle/_ref/libarcos_ref_dropin.so): the reference without its
  Fortran wrapper; cdr_advect_diffu (src/cdr.c:945-949) calls the device's
  arcos_cdr_advect_vec for every grid, species and stage.  Everything else
  is the reference's code, so results are bit-identical, dt included, for
  any tree and any number of steps.
* Grid route (oracle/_ref/libarcos_ref_adapter.so): the reference with its
  cdr_rk2 renamed, and arcos_b200/adapter/cdr_grid_adapter.c providing
  cdr_rk2(cdr_grid_t *, h, t) on the device (the tree, the model and the
  field solve stay the reference's, on the host).  Exact arithmetic, so
  bit-identical too; on trees the comparison is with the reference's step
  on a freshly cloned tree (every child's d_dens starts at zero, as
  cdr_update_refined gives it in a real run, src/cdr.c:1363-1376).

Both libraries are built by oracle/Makefile where the reference sources
are present; elsewhere these tests are skipped.
"""
import copy

import numpy as np
import pytest

from arcos_b200 import workloads
from oracle import bind
from parity_util import max_ulp

pytestmark = pytest.mark.gpu

needs_dropin = pytest.mark.skipif(not (bind.ref_available("dropin") and bind.ref_available("plain")),
                                  reason="reference build absent")
needs_adapter = pytest.mark.skipif(not (bind.ref_available("adapter") and bind.ref_available("plain")),
                                   reason="reference build absent")


def ref_tree(pb, variant, field_mode=bind.FIELD_FIXED):
    t = bind.RefTree(copy.deepcopy(pb.params), pb.model, pb.specs, field_mode=field_mode, omp=variant)
    for g, per in enumerate(pb.dens):
        for s, a in enumerate(per):
            t.dens(g, s)[...] = a
    if field_mode == bind.FIELD_FIXED:
        for g, (er, ez, et) in enumerate(pb.fields):
            t.set_fixed_field(g, er, ez, et if et is not None else pb.specs[g].zeros())
    return t


def assert_bitwise(a, b, pb, what=("dens", "d_dens")):
    for g in range(len(pb.specs)):
        for w in what:
            for s in range(pb.model.no_species if w in ("dens", "d_dens") else 1):
                x, y = a.array(g, w, s), b.array(g, w, s)
                assert max_ulp(x, y) == 0, (g, w, s, max_ulp(x, y))


def small_tree():
    return workloads.amr(n_patches=10, levels=3, root_nr=32, root_nz=64, side_lo=8, side_hi=24, seed=2)


# ---------------------------------------------------------------- seam ----
@needs_dropin
@pytest.mark.parametrize("field", ["uniform", "wavy"])
def test_seam_route_single_grid(cuda_device, field):
    pb = workloads.plain(nr=40, nz=72, ion_mass=1.0, noise=1e-3, seed=3, field=field)
    ref, dev = ref_tree(pb, "plain"), ref_tree(pb, "dropin")
    for _ in range(4):
        assert ref.rk2(50.0) == dev.rk2(50.0)
    assert_bitwise(ref, dev, pb)


@needs_dropin
def test_seam_route_tree(cuda_device):
    pb = small_tree()
    ref, dev = ref_tree(pb, "plain"), ref_tree(pb, "dropin")
    for _ in range(3):
        assert ref.rk2(50.0) == dev.rk2(50.0)
    assert_bitwise(ref, dev, pb)


@needs_dropin
def test_seam_route_field_in_loop(cuda_device):
    pb = workloads.plain(nr=32, nz=64, ion_mass=0.0, seed=9)
    ref = ref_tree(pb, "plain", bind.FIELD_POISSON)
    dev = ref_tree(pb, "dropin", bind.FIELD_POISSON)
    ref.call("ref_calc_charge_r")
    dev.call("ref_calc_charge_r")
    for _ in range(3):
        assert ref.rk2(50.0) == dev.rk2(50.0)
    assert_bitwise(ref, dev, pb, ("dens", "d_dens", "charge", "er", "ez"))


# ---------------------------------------------------------------- grid ----
@needs_adapter
@pytest.mark.parametrize("field", ["uniform", "wavy"])
@pytest.mark.parametrize("ion_mass", [0.0, 1.0])
def test_grid_route_single_grid(cuda_device, field, ion_mass):
    pb = workloads.plain(nr=40, nz=72, ion_mass=ion_mass, noise=1e-3, seed=5, field=field)
    ref, dev = ref_tree(pb, "plain"), ref_tree(pb, "adapter")
    ref.call("ref_calc_charge_r")
    dev.call("ref_calc_charge_r")
    for _ in range(4):
        assert ref.rk2(50.0) == dev.rk2(50.0)
    assert_bitwise(ref, dev, pb, ("dens", "d_dens", "charge", "er", "ez", "eabs"))


@needs_adapter
def test_grid_route_field_in_loop(cuda_device):
    """The reference's own host field solve between the device stages."""
    pb = workloads.plain(nr=32, nz=64, ion_mass=0.0, seed=9)
    ref = ref_tree(pb, "plain", bind.FIELD_POISSON)
    dev = ref_tree(pb, "adapter", bind.FIELD_POISSON)
    ref.call("ref_calc_charge_r")
    dev.call("ref_calc_charge_r")
    for _ in range(3):
        assert ref.rk2(50.0) == dev.rk2(50.0)
    assert_bitwise(ref, dev, pb, ("dens", "d_dens", "charge", "er", "ez", "eabs"))


@needs_adapter
def test_grid_route_theta(cuda_device):
    pb = workloads.plain(nr=20, nz=36, ntheta=4, ion_mass=1.0, noise=1e-6, seed=3, field="wavy")
    pb.params.per_plane = False
    ref, dev = ref_tree(pb, "plain"), ref_tree(pb, "adapter")
    ref.call("ref_calc_charge_r")
    dev.call("ref_calc_charge_r")
    for _ in range(3):
        assert ref.rk2(50.0) == dev.rk2(50.0)
    assert_bitwise(ref, dev, pb, ("dens", "charge"))


@needs_adapter
def test_grid_route_tree(cuda_device):
    pb = small_tree()
    ref, dev = ref_tree(pb, "plain"), ref_tree(pb, "adapter")
    ref.call("ref_calc_charge_r")
    dev.call("ref_calc_charge_r")
    for _ in range(3):
        # the reference's step on a freshly cloned tree (children's d_dens zeroed)
        h_ref = ref.rk2_sw(50.0, per_plane=False, zero_all=True)
        assert h_ref == dev.rk2(50.0)
    assert_bitwise(ref, dev, pb, ("dens", "d_dens", "charge"))


@needs_adapter
def test_grid_route_keeps_context_across_calls_and_rebuilds_on_change(cuda_device):
    """Two trees of different shapes through the same adapter, one after the
    other (as a refinement would change the tree), each matching the
    reference."""
    for pb in (workloads.plain(nr=24, nz=40, ion_mass=1.0, noise=1e-3, seed=1),
               workloads.plain(nr=32, nz=48, ion_mass=1.0, noise=1e-3, seed=2, field="wavy")):
        ref, dev = ref_tree(pb, "plain"), ref_tree(pb, "adapter")
        ref.call("ref_calc_charge_r")
        dev.call("ref_calc_charge_r")
        for _ in range(2):
            assert ref.rk2(50.0) == dev.rk2(50.0)
        assert_bitwise(ref, dev, pb, ("dens", "charge"))
        del ref, dev
