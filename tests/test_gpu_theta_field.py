"""The device field solve on 3-D grids (poisson_kernel.cuh: the charge to
theta modes, one Helmholtz solve per mode with lambda = -w2k[m], the field
back with hc2r and dft_diff; cdr_calc_field_r, src/cdr.c:532-580) against
the oracle's restatement (oracle/poisson_host.c oracle_theta_field with
oracle/dft_host.c), which test_theta_field.py pins bit for bit to the
reference's own dft.c and cdr_calc_field_r.  The device evaluates every sum
in the oracle's order from host tables, so everything is bit-identical:
the single solve, and the field-in-the-loop steps with their dt.
"""
import numpy as np
import pytest

from arcos_b200 import workloads
from arcos_b200.cdr import CdrTree
from oracle import bind
from parity_util import max_ulp, port_tree, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nt", [2, 4, 5, 8, 16])
def test_device_theta_field_bitwise_equals_oracle(cuda_device, nt):
    nr, nz = 24, 40
    pb = workloads.plain(nr=nr, nz=nz, ntheta=nt, ion_mass=0.0, noise=1e-3, seed=4)
    pb.params.E0_z = 0.0                        # the raw solve, no applied field
    dev = CdrTree(pb.params, pb.model, pb.specs, exact=True)
    rng = np.random.default_rng(nt)
    charge = pb.specs[0].zeros()
    charge[2:-2, 2:-2, 2:-2] = rng.normal(size=(nt, nz, nr)) * 1e-2
    dev.upload(0, "charge", charge)
    dev.set_field_poisson(True)
    dev.solve_field(0)
    ch_h, er_h, ez_h, et_h = bind.theta_field(nr, nz, nt, pb.params.dr(0), pb.params.dz(0), charge)
    real = slice(2, nt + 2)
    assert max_ulp(dev.download(0, "charge")[real], ch_h[real]) == 0
    for w, h in (("er", er_h), ("ez", ez_h), ("etheta", et_h)):
        d = dev.download(0, w)
        assert max_ulp(d[real], h[real]) == 0, w
        # the theta ghost planes are the periodic copies (cdr_set_periodic)
        assert np.array_equal(d[0], d[nt]) and np.array_equal(d[1], d[nt + 1])
        assert np.array_equal(d[nt + 2], d[2]) and np.array_equal(d[nt + 3], d[3])
    assert np.max(np.abs(et_h[real])) > 0
    dev.close()


@pytest.mark.parametrize("nt,per_plane", [(4, True), (4, False), (8, True)])
def test_device_3d_field_in_loop_matches_oracle(cuda_device, nt, per_plane):
    """The field solved on the device at both stages of every step, replayed
    from the step graph, against the oracle with the same solve on the host:
    the same dt and densities bit for bit (exact mode), and the same field."""
    pb = workloads.plain(nr=24, nz=40, ntheta=nt, ion_mass=0.0, noise=0.3, seed=11)
    pb.params.per_plane = per_plane
    port = port_tree(pb, field_mode=bind.FIELD_POISSON, per_plane=per_plane)
    port.call("port_calc_charge")
    dts_p = np.array([port.rk2(50.0)[0] for _ in range(6)])
    dev = CdrTree(pb.params, pb.model, pb.specs, exact=True)
    for s in range(2):
        dev.upload(0, "dens", pb.dens[0][s], s)
    dev.cdr_calc_charge_r(0)
    dev.set_field_poisson(True)
    dts_d = dev.run(6, 50.0)[0]
    assert np.array_equal(dts_d, dts_p), (dts_d, dts_p)
    for s in range(2):
        a, b = dev.download(0, "dens", s), port.dens(0, s)
        assert max_ulp(a, b) == 0, (s, rel_err(a, b))
    real = slice(2, nt + 2)
    for w in ("er", "ez", "etheta", "eabs"):
        assert max_ulp(dev.download(0, w)[real], port.array(0, w, 0)[real]) == 0, w
    dev.close()


def test_device_3d_field_step_by_step_and_tree_entry(cuda_device):
    """One step per call, and the grid-level cdr_rk2 entry, on the 3-D solve."""
    nt = 4
    pb = workloads.plain(nr=20, nz=36, ntheta=nt, ion_mass=0.0, noise=0.3, seed=5)
    pb.params.per_plane = True
    port = port_tree(pb, field_mode=bind.FIELD_POISSON, per_plane=True)
    port.call("port_calc_charge")
    dev = CdrTree(pb.params, pb.model, pb.specs, exact=True)
    for s in range(2):
        dev.upload(0, "dens", pb.dens[0][s], s)
    dev.cdr_calc_charge_r(0)
    dev.set_field_poisson(True)
    for _ in range(2):
        assert dev.run(1, 50.0)[0][0] == port.rk2(50.0)[0]
    for _ in range(2):
        assert dev.cdr_rk2(50.0) == port.rk2(50.0)[0]
    for s in range(2):
        assert max_ulp(dev.download(0, "dens", s), port.dens(0, s)) == 0
    dev.close()


def test_device_3d_field_in_loop_division_free_within_tolerance(cuda_device):
    """The default (division-free) stage kernels with the 3-D field solved
    on the device: within 1e-12 of the oracle per step (resynchronised to
    the oracle after every step; the field solve itself is exact)."""
    nt = 4
    pb = workloads.plain(nr=24, nz=40, ntheta=nt, ion_mass=0.0, noise=0.3, seed=13)
    port = port_tree(pb, field_mode=bind.FIELD_POISSON, per_plane=True)
    port.call("port_calc_charge")
    dev = CdrTree(pb.params, pb.model, pb.specs, exact=False)
    for s in range(2):
        dev.upload(0, "dens", pb.dens[0][s], s)
    dev.cdr_calc_charge_r(0)
    dev.set_field_poisson(True)
    for _ in range(4):
        hp = port.rk2(50.0)[0]
        hd = dev.run(1, 50.0)[0][0]
        assert abs(hd - hp) <= 1e-12 * hp
        for s in range(2):
            a, b = dev.download(0, "dens", s), port.dens(0, s)
            assert rel_err(a, b) <= 1e-12, (s, rel_err(a, b))
            dev.upload(0, "dens", b, s)
        dev.cdr_calc_charge_r(0)
    dev.close()
