"""Device path against the CPU oracle (oracle/cdr_port.c, itself pinned to the
reference sources in test_oracle_pin.py) on the same seeded inputs.

The bar is the north-star tolerance, 1e-12 relative per step; with FMA
contraction disabled the device arithmetic is the reference's operation for
operation, so the tests also report (and bound) the ulp distance.
"""
import numpy as np
import pytest

from arcos_b200 import workloads
from arcos_b200.cdr import CdrTree, cdr_advect_vec
from oracle import bind
from parity_util import max_ulp, port_tree, rel_err, single_family

pytestmark = pytest.mark.gpu

TOL = 1e-12


def device_tree(pb, exact=True, **kw):
    t = CdrTree(pb.params, pb.model, pb.specs, exact=exact, **kw)
    for g, per in enumerate(pb.dens):
        for s, a in enumerate(per):
            t.upload(g, "dens", a, s)
    for f, E in enumerate(pb.family_E):
        t.set_family_field(f, *E)
    t.set_fixed_field(pb.fields)
    return t


def compare_state(dev, port, pb, gids=None, what="dens"):
    worst = 0.0
    for g in (gids if gids is not None else range(len(pb.specs))):
        for s in range(pb.model.no_species):
            a = dev.download(g, what, s)
            b = port.array(g, what, s)
            worst = max(worst, rel_err(a, b))
            assert rel_err(a, b) <= TOL, (g, s, rel_err(a, b), max_ulp(a, b))
    return worst


@pytest.mark.parametrize("ion_mass", [0.0, 1.0])
def test_fused_run_matches_oracle(cuda_device, ion_mass):
    pb = workloads.plain(nr=40, nz=72, ion_mass=ion_mass, noise=1e-3, seed=3)
    port = port_tree(pb)
    dev = device_tree(pb)
    dts_p = [port.rk2(50.0)[0] for _ in range(6)]
    dts_d = dev.run(6, 50.0)[0]
    assert np.array_equal(dts_d, np.array(dts_p)), (dts_d, dts_p)
    compare_state(dev, port, pb)
    for s in range(2):
        assert max_ulp(dev.download(0, "dens", s), port.dens(0, s)) == 0


@pytest.mark.parametrize("ion_mass", [0.0, 1.0])
def test_general_step_matches_oracle(cuda_device, ion_mass):
    pb = workloads.plain(nr=36, nz=64, ion_mass=ion_mass, noise=1e-3, seed=5)
    port = port_tree(pb)
    dev = device_tree(pb)
    for _ in range(4):
        hp, st = port.rk2(50.0)
        hd = dev.cdr_rk2(50.0)
        assert st == 0 and hd == hp
    compare_state(dev, port, pb)
    compare_state(dev, port, pb, what="d_dens")


def test_dirichlet_and_odd_sizes(cuda_device):
    pb = workloads.plain(nr=45, nz=51, ion_mass=1.0, noise=1e-3, seed=7)
    pb.params.cdr_bnd_top = -1
    pb.params.cdr_bnd_right = -1
    port = port_tree(pb)
    dev = device_tree(pb)
    dts_p = [port.rk2(50.0)[0] for _ in range(3)]
    dts_d = dev.run(3, 50.0)[0]
    assert np.array_equal(dts_d, np.array(dts_p))
    compare_state(dev, port, pb)


@pytest.mark.parametrize("per_plane", [True, False])
def test_theta_planes(cuda_device, per_plane):
    pb = workloads.plain(nr=24, nz=40, ntheta=4, ion_mass=1.0, noise=1e-6, seed=11)
    pb.params.per_plane = per_plane
    port = port_tree(pb)
    dev = device_tree(pb)
    dts_p = [port.rk2(50.0)[0] for _ in range(3)]
    dts_d = dev.run(3, 50.0)[0]
    assert np.array_equal(dts_d, np.array(dts_p))
    compare_state(dev, port, pb)


def test_amr_tree(cuda_device):
    pb = workloads.amr(n_patches=12, levels=3, root_nr=32, root_nz=64, side_lo=8, side_hi=24, seed=2)
    assert len(pb.specs) >= 6
    port = port_tree(pb, zero_all=True)
    dev = device_tree(pb)
    for _ in range(3):
        hp, st = port.rk2(50.0)
        hd = dev.cdr_rk2(50.0)
        assert st == 0 and hd == hp
    compare_state(dev, port, pb)


@pytest.mark.parametrize("tile", [0, 1, 2, 3, 4, 5])
@pytest.mark.parametrize("field", ["uniform", "wavy"])
def test_amr_tree_lean_batched_step(cuda_device, tile, field):
    """The lean batched tree step (the fused stage kernels over every patch,
    tiled or marching, ghosts from prepare_grid) per step against the oracle
    at 1e-12; also 3 steps replayed from the step graph in one call."""
    pb = workloads.amr(n_patches=12, levels=3, root_nr=32, root_nz=64, side_lo=8, side_hi=24, seed=2)
    if field == "wavy":
        pb.fields = [workloads.wavy_field(sp, pb.params, seed=50 + g) for g, sp in enumerate(pb.specs)]
    port = port_tree(pb, zero_all=True)
    dev = device_tree(pb, exact=False)
    dev.set_tile(tile)
    for _ in range(3):
        hp = port.rk2(50.0)[0]
        hd = dev.run(1, 50.0)[0][0]
        assert abs(hd - hp) <= TOL * hp
        for g in range(len(pb.specs)):
            for s in range(2):
                a, b = dev.download(g, "dens", s), port.dens(g, s)
                assert rel_err(a, b) <= TOL, (tile, g, s, rel_err(a, b))
                dev.upload(g, "dens", b, s)
    dts_p = [port.rk2(50.0)[0] for _ in range(3)]
    dts_d = dev.run(3, 50.0)[0]
    assert rel_err(dts_d, np.array(dts_p)) <= TOL
    compare_state(dev, port, pb)


def test_amr_per_patch_mode_identical(cuda_device):
    pb = workloads.amr(n_patches=10, levels=3, root_nr=32, root_nz=64, side_lo=8, side_hi=24, seed=4)
    a = device_tree(pb)
    b = device_tree(pb, per_patch=True)
    for _ in range(2):
        assert a.cdr_rk2(50.0) == b.cdr_rk2(50.0)
    for g in range(len(pb.specs)):
        for s in range(2):
            assert np.array_equal(a.download(g, "dens", s), b.download(g, "dens", s))


def test_field_in_loop(cuda_device):
    pb = workloads.plain(nr=32, nz=64, ion_mass=0.0, seed=9)
    port = port_tree(pb, field_mode=bind.FIELD_POISSON)
    port.call("port_calc_charge")
    dev = CdrTree(pb.params, pb.model, pb.specs, exact=True)
    for s in range(2):
        dev.upload(0, "dens", pb.dens[0][s], s)
    dev.cdr_calc_charge_r(0)
    sp = pb.specs[0]
    dr, dz = pb.params.dr(0), pb.params.dz(0)

    def field(stage, charge):
        er, ez = bind.poisson_field(sp.nr, sp.nz, dr, dz, charge)
        return er, ez, None

    dev.set_field_callback(field)
    dts_p = [port.rk2(50.0)[0] for _ in range(3)]
    dts_d = dev.run(3, 50.0)[0]
    assert np.allclose(dts_d, dts_p, rtol=TOL, atol=0)
    compare_state(dev, port, pb)


def test_kinetic_batch(cuda_device):
    pb = workloads.kinetic_batch(n_inst=3, points=200, sizes_r=(24, 40), sizes_z=(32, 48), seed=1)
    dev = device_tree(pb)
    dts_d = dev.run(3, 50.0)
    for i in range(3):
        sub = single_family(pb, i)
        port = port_tree(sub, E=pb.family_E[i])
        dts_p = [port.rk2(50.0)[0] for _ in range(3)]
        assert np.array_equal(dts_d[i], np.array(dts_p)), (i, dts_d[i], dts_p)
        for s in range(6):
            a = dev.download(i, "dens", s)
            b = port.dens(0, s)
            assert rel_err(a, b) <= TOL, (i, s, rel_err(a, b))


def test_narrow_seam(cuda_device):
    rng = np.random.default_rng(0)
    r0, r1, z0, z1 = 6, 30, 0, 20
    shape = (z1 - z0 + 4, r1 - r0 + 4)
    dens = rng.random(shape) ** 3
    dens[:, 5] = dens[:, 6]                       # flat stretches hit the |dC| mask
    er = rng.normal(size=shape)
    ez = rng.normal(size=shape)
    d0 = rng.normal(size=shape)
    d_dev = d0.copy()
    d_port = d0.copy()
    cdr_advect_vec(1.0, -1.0, dens, d_dev, er, ez, 0.1, 1 / 64, 1 / 64, r0, r1, z0, z1)
    lib = bind.port_lib()
    P = bind._dp
    lib.port_advect_vec(1.0, -1.0, P(dens), P(d_port), P(er), P(ez), 0.1, 1 / 64, 1 / 64,
                        r0, r1, z0, z1)
    assert max_ulp(d_dev, d_port) == 0


@pytest.mark.parametrize("ntheta", [1, 4])
def test_fast_limiter_within_tolerance(cuda_device, ntheta):
    """The division-free limiter (the default) against the oracle: 1e-12
    relative per step, the north-star tolerance."""
    pb = workloads.plain(nr=40, nz=72, ntheta=ntheta, ion_mass=1.0, noise=1e-3, seed=13)
    port = port_tree(pb)
    dev = device_tree(pb, exact=False)
    for _ in range(5):
        hp = port.rk2(50.0)[0]
        hd = dev.run(1, 50.0)[0][0]
        assert abs(hd - hp) <= TOL * hp
        for s in range(2):
            a, b = dev.download(0, "dens", s), port.dens(0, s)
            assert rel_err(a, b) <= TOL, rel_err(a, b)
            # resynchronise so the check is per step
            dev.upload(0, "dens", b, s)


def test_fast_limiter_long_run(cuda_device):
    """1000 steps with the division-free limiter stay within 1e-9 of the oracle."""
    pb = workloads.plain(nr=32, nz=64, ion_mass=1.0, noise=1e-3, seed=17)
    port = port_tree(pb)
    dev = device_tree(pb, exact=False)
    for _ in range(1000):
        port.rk2(50.0)
    dev.run(1000, 50.0)
    for s in range(2):
        a, b = dev.download(0, "dens", s), port.dens(0, s)
        assert rel_err(a, b) <= 1e-9, rel_err(a, b)


@pytest.mark.parametrize("tile", [0, 1, 2, 3, 4, 5])
@pytest.mark.parametrize("ntheta", [1, 4])
def test_fused_every_tile_shape(cuda_device, tile, ntheta):
    """The fused step (division-free limiter) with each tile shape the
    autotuner can pick, per step against the oracle at 1e-12, then four
    steps replayed from the step graph."""
    pb = workloads.plain(nr=40, nz=72, ntheta=ntheta, ion_mass=1.0, noise=1e-3, seed=21)
    port = port_tree(pb)
    dev = device_tree(pb, exact=False)
    dev.set_tile(tile)
    for _ in range(3):
        hp = port.rk2(50.0)[0]
        hd = dev.run(1, 50.0)[0][0]
        assert abs(hd - hp) <= TOL * hp
        for s in range(2):
            a, b = dev.download(0, "dens", s), port.dens(0, s)
            assert rel_err(a, b) <= TOL, (tile, s, rel_err(a, b))
            dev.upload(0, "dens", b, s)
    for _ in range(4):
        port.rk2(50.0)
    dev.run(4, 50.0)
    for s in range(2):
        assert rel_err(dev.download(0, "dens", s), port.dens(0, s)) <= 4 * TOL


@pytest.mark.parametrize("tile", [0, 1, 2, 3, 4, 5])
def test_kinetic_batch_fused_every_tile_shape(cuda_device, tile):
    """Six species, nine reactions, three families of different sizes on the
    fused path with each tile shape, per step against the oracle at 1e-12."""
    pb = workloads.kinetic_batch(n_inst=3, points=200, sizes_r=(24, 40), sizes_z=(32, 48), seed=1)
    dev = device_tree(pb, exact=False)
    dev.set_tile(tile)
    ports = [port_tree(single_family(pb, i), E=pb.family_E[i]) for i in range(3)]
    for _ in range(3):
        hd = dev.run(1, 50.0)
        for i, port in enumerate(ports):
            hp = port.rk2(50.0)[0]
            assert abs(hd[i][0] - hp) <= TOL * hp
            for s in range(6):
                a, b = dev.download(i, "dens", s), port.dens(0, s)
                assert rel_err(a, b) <= TOL, (tile, i, s, rel_err(a, b))
                dev.upload(i, "dens", b, s)
