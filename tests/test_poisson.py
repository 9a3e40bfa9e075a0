"""The field solve on the device (poisson_kernel.cuh, the pois_solve_a seam
of src/poisson.c:763-767) against the host solver that both sides use at that
seam in the other tests (oracle/poisson_host.c: hstcyl's 5-point cylindrical
operator, regular axis, Dirichlet on r = L_r, z = 0, z = L_z).  The device
evaluates every sum in the host solver's order from host-evaluated
coefficients, so the fields must be bit-identical; FISHPACK itself cannot
be built here, so the solver is not pinned to FISHPACK.
"""
import numpy as np
import pytest

from arcos_b200 import workloads
from arcos_b200.cdr import CdrTree
from oracle import bind
from parity_util import max_ulp, port_tree, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape", [(32, 64), (45, 51), (128, 256)])
def test_device_field_bitwise_equals_host_solver(cuda_device, shape):
    nr, nz = shape
    pb = workloads.plain(nr=nr, nz=nz, ion_mass=0.0, noise=1e-3, seed=4)
    pb.params.E0_z = 0.0                        # the raw solve, no applied field
    dev = CdrTree(pb.params, pb.model, pb.specs, exact=True)
    rng = np.random.default_rng(nr + nz)
    charge = pb.specs[0].zeros()
    charge[0, 2:-2, 2:-2] = rng.normal(size=(nz, nr)) * 1e-2
    dev.upload(0, "charge", charge)
    dev.set_field_poisson(True)
    dev.solve_field(0)
    er_h, ez_h = bind.poisson_field(nr, nz, pb.params.dr(0), pb.params.dz(0), charge)
    er_d, ez_d = dev.download(0, "er"), dev.download(0, "ez")
    assert max_ulp(er_d[0], er_h) == 0
    assert max_ulp(ez_d[0], ez_h) == 0
    dev.close()


def test_c0_field_in_loop_on_device_200_steps(cuda_device):
    """c0 (128 x 256, immobile ions) with the field solved on the device at
    both stages of every step, 200 steps replayed from the step graph, the
    reference's arithmetic (exact mode): the same densities and dt as the
    oracle with the host solver in the loop."""
    pb = workloads.plain(nr=128, nz=256, ion_mass=0.0, seed=0)
    port = port_tree(pb, field_mode=bind.FIELD_POISSON)
    port.call("port_calc_charge")
    dts_p = np.array([port.rk2(50.0)[0] for _ in range(200)])
    dev = CdrTree(pb.params, pb.model, pb.specs, exact=True)
    for s in range(2):
        dev.upload(0, "dens", pb.dens[0][s], s)
    dev.cdr_calc_charge_r(0)
    dev.set_field_poisson(True)
    dts_d = dev.run(200, 50.0)[0]
    assert np.array_equal(dts_d, dts_p), float(np.max(np.abs(dts_d - dts_p) / dts_p))
    for s in range(2):
        a, b = dev.download(0, "dens", s), port.dens(0, s)
        assert max_ulp(a, b) == 0, (s, rel_err(a, b))
    dev.close()


def test_device_field_per_step_matches_callback(cuda_device):
    """The device solve and the host callback give the same steps."""
    pb = workloads.plain(nr=32, nz=64, ion_mass=1.0, noise=1e-3, seed=9)
    sp = pb.specs[0]
    dr, dz = pb.params.dr(0), pb.params.dz(0)
    a = CdrTree(pb.params, pb.model, pb.specs, exact=True)
    b = CdrTree(pb.params, pb.model, pb.specs, exact=True)
    for t in (a, b):
        for s in range(2):
            t.upload(0, "dens", pb.dens[0][s], s)
        t.cdr_calc_charge_r(0)
    a.set_field_poisson(True)
    b.set_field_callback(lambda stage, ch: (*bind.poisson_field(sp.nr, sp.nz, dr, dz, ch), None))
    for _ in range(4):
        assert np.array_equal(a.run(1, 50.0), b.run(1, 50.0))
    for s in range(2):
        assert np.array_equal(a.download(0, "dens", s), b.download(0, "dens", s))
    # and through the grid-level cdr_rk2
    assert a.cdr_rk2(50.0) == b.cdr_rk2(50.0)
    a.close()
    b.close()


def test_device_field_refuses_trees_and_callbacks(cuda_device):
    pb = workloads.amr(n_patches=6, levels=2, root_nr=32, root_nz=64, side_lo=8, side_hi=16, seed=1)
    t = CdrTree(pb.params, pb.model, pb.specs)
    with pytest.raises(Exception):
        t.set_field_poisson(True)
    t.close()
