"""Device path against the CPU oracle on a non-uniform fixed field
(``workloads.wavy_field``): both field components change sign inside a
tile, and |E| sweeps the whole reaction table, from underflow to overflow.

This is what exercises, on the device, the radial drift of every kernel
(the Koren limiter on radial faces with the psi = -1 mask, .f90:233-308),
the per-lane mixed upwind orientation where the field changes sign inside
a warp, the tile's right-boundary faces, and the table lookup k(|E|) at
many nodes (reaction.c:127-142) - all multiplied by zero, or evaluated at
a single |E|, under the uniform applied field of the other parity tests.

Tolerances: exact mode bit for bit (and the dt sequence identical); the
division-free limiter 1e-12 relative per step (resynchronised to the
oracle after every step) and 1e-9 after 1000 steps.
"""
import numpy as np
import pytest

from arcos_b200 import workloads
from parity_util import max_ulp, port_tree, rel_err, single_family
from test_gpu_parity import compare_state, device_tree

pytestmark = pytest.mark.gpu

TOL = 1e-12


def wavy(nr=40, nz=72, ntheta=1, seed=13, ion_mass=1.0):
    return workloads.plain(nr=nr, nz=nz, ntheta=ntheta, ion_mass=ion_mass, noise=1e-3, seed=seed,
                           field="wavy")


@pytest.mark.parametrize("ion_mass", [0.0, 1.0])
def test_exact_run_bitwise_on_wavy_field(cuda_device, ion_mass):
    pb = wavy(ion_mass=ion_mass, seed=3)
    port = port_tree(pb)
    dev = device_tree(pb)
    dts_p = [port.rk2(50.0)[0] for _ in range(6)]
    dts_d = dev.run(6, 50.0)[0]
    assert np.array_equal(dts_d, np.array(dts_p)), (dts_d, dts_p)
    for s in range(2):
        assert max_ulp(dev.download(0, "dens", s), port.dens(0, s)) == 0


def test_general_step_on_wavy_field(cuda_device):
    """The tree-form step (cdr_rk2 entry point, d_dens materialised)."""
    pb = wavy(nr=36, nz=64, seed=5)
    port = port_tree(pb)
    dev = device_tree(pb)
    for _ in range(4):
        hp, st = port.rk2(50.0)
        assert st == 0 and dev.cdr_rk2(50.0) == hp
    compare_state(dev, port, pb)
    compare_state(dev, port, pb, what="d_dens")


@pytest.mark.parametrize("ntheta", [1, 4])
def test_fast_limiter_per_step_on_wavy_field(cuda_device, ntheta):
    pb = wavy(ntheta=ntheta)
    port = port_tree(pb)
    dev = device_tree(pb, exact=False)
    for _ in range(5):
        hp = port.rk2(50.0)[0]
        hd = dev.run(1, 50.0)[0][0]
        assert abs(hd - hp) <= TOL * hp
        for s in range(2):
            a, b = dev.download(0, "dens", s), port.dens(0, s)
            assert rel_err(a, b) <= TOL, (s, rel_err(a, b))
            dev.upload(0, "dens", b, s)


@pytest.mark.parametrize("tile", [0, 1, 2, 3, 4, 5])
@pytest.mark.parametrize("ntheta", [1, 4])
def test_fused_every_tile_shape_on_wavy_field(cuda_device, tile, ntheta):
    pb = wavy(ntheta=ntheta, seed=21)
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


def test_fast_limiter_long_run_on_wavy_field(cuda_device):
    """1000 steps of the division-free limiter stay within 1e-9 of the oracle."""
    pb = wavy(nr=32, nz=64, seed=17)
    port = port_tree(pb)
    dev = device_tree(pb, exact=False)
    dts_p = np.array([port.rk2(50.0)[0] for _ in range(1000)])
    dts_d = dev.run(1000, 50.0)[0]
    assert rel_err(dts_d, dts_p) <= 1e-9
    for s in range(2):
        a, b = dev.download(0, "dens", s), port.dens(0, s)
        assert rel_err(a, b) <= 1e-9, rel_err(a, b)


@pytest.mark.parametrize("tile", [0, 1, 2, 3, 4, 5])
def test_kinetic_batch_on_wavy_field(cuda_device, tile):
    """Six species, nine reactions, three families with their own applied
    fields, each tile shape; on these short instances |E| stays near each
    family's applied field (a few adjacent nodes of the 200-node tables)."""
    pb = workloads.kinetic_batch(n_inst=3, points=200, sizes_r=(24, 40), sizes_z=(32, 48), seed=1,
                                 field="wavy")
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


@pytest.mark.parametrize("tile", [0, 2, 3])
def test_kinetic_batch_on_full_sweep_field(cuda_device, tile):
    """The same on ``field="wavy_full"``: every instance's |E| runs from below
    the tables' first node to above their last, so the division-free
    kernel's lookups of all nine reactions are compared at both sentinel
    nodes and across the table."""
    pb = workloads.kinetic_batch(n_inst=3, points=200, sizes_r=(24, 40), sizes_z=(32, 48), seed=1,
                                 field="wavy_full")
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


def test_kinetic_batch_exact_on_wavy_field(cuda_device):
    pb = workloads.kinetic_batch(n_inst=3, points=200, sizes_r=(24, 40), sizes_z=(32, 48), seed=2,
                                 field="wavy")
    dev = device_tree(pb)
    dts_d = dev.run(3, 50.0)
    for i in range(3):
        port = port_tree(single_family(pb, i), E=pb.family_E[i])
        dts_p = [port.rk2(50.0)[0] for _ in range(3)]
        assert np.array_equal(dts_d[i], np.array(dts_p)), (i, dts_d[i], dts_p)
        for s in range(6):
            a, b = dev.download(i, "dens", s), port.dens(0, s)
            assert rel_err(a, b) <= TOL, (i, s, rel_err(a, b))
