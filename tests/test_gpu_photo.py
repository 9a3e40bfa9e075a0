"""Photoionization on the device (poisson_kernel.cuh k_photo_*, one
Helmholtz solve per term and theta mode, arcos_set_photo) against the
oracle's photo_calc (oracle/cdr_port.c), which test_photo.py pins bit for
bit to the reference's own photo.c.  Exact mode: every density and dt
bit-identical; the division-free step within 1e-12 per step.
"""
import numpy as np
import pytest

from arcos_b200 import workloads
from arcos_b200.cdr import CdrTree
from oracle import bind
from parity_util import max_ulp, port_tree, rel_err
from test_gpu_parity import device_tree

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ntheta,field", [(1, "uniform"), (1, "wavy"), (4, "uniform")])
def test_device_photo_run_bitwise(cuda_device, ntheta, field):
    pb = workloads.photo(nr=24, nz=40, ntheta=ntheta, noise=0.3, seed=3, field=field)
    port = port_tree(pb, per_plane=True)
    dts_p = np.array([port.rk2(50.0)[0] for _ in range(5)])
    dev = device_tree(pb, exact=True)
    dts_d = dev.run(5, 50.0)[0]
    assert np.array_equal(dts_d, dts_p), (dts_d, dts_p)
    for s in range(pb.model.no_species):
        a, b = dev.download(0, "dens", s), port.dens(0, s)
        assert max_ulp(a, b) == 0, (s, rel_err(a, b))
    assert np.max(dev.download(0, "dens", 4)) > 0          # the photo ions
    dev.close()


def test_device_photo_tree_entry_and_pieces(cuda_device):
    """The grid-level cdr_rk2 and the derivative entry points with photo."""
    pb = workloads.photo(nr=20, nz=36, noise=0.3, seed=5)
    port = port_tree(pb)
    dev = device_tree(pb, exact=True)
    for _ in range(3):
        assert dev.cdr_rk2(50.0) == port.rk2(50.0)[0]
    for w in ("dens", "d_dens"):
        for s in range(pb.model.no_species):
            assert max_ulp(dev.download(0, w, s), port.array(0, w, s)) == 0, (w, s)
    # cdr_calc_d_dens alone (reactions, photo_calc, drift/diffusion)
    dev.cdr_calc_d_dens(0)
    port.call("port_calc_d_dens")
    for s in range(pb.model.no_species):
        assert max_ulp(dev.download(0, "d_dens", s), port.array(0, "d_dens", s)) == 0, s
    dev.close()


@pytest.mark.parametrize("ntheta", [1, 4])
def test_device_photo_with_device_field_in_loop(cuda_device, ntheta):
    pb = workloads.photo(nr=24, nz=40, ntheta=ntheta, noise=0.3, seed=7)
    port = port_tree(pb, field_mode=bind.FIELD_POISSON, per_plane=True)
    port.call("port_calc_charge")
    dts_p = np.array([port.rk2(50.0)[0] for _ in range(4)])
    dev = CdrTree(pb.params, pb.model, pb.specs, exact=True)
    for s in range(pb.model.no_species):
        dev.upload(0, "dens", pb.dens[0][s], s)
    dev.cdr_calc_charge_r(0)
    dev.set_field_poisson(True)
    dts_d = dev.run(4, 50.0)[0]
    assert np.array_equal(dts_d, dts_p), (dts_d, dts_p)
    for s in range(pb.model.no_species):
        assert max_ulp(dev.download(0, "dens", s), port.dens(0, s)) == 0, s
    dev.close()


def test_device_photo_fast_step_within_tolerance(cuda_device):
    pb = workloads.photo(nr=32, nz=48, noise=0.3, seed=9, field="wavy")
    port = port_tree(pb)
    dev = device_tree(pb, exact=False)
    for _ in range(4):
        hp = port.rk2(50.0)[0]
        hd = dev.run(1, 50.0)[0][0]
        assert abs(hd - hp) <= 1e-12 * hp
        for s in range(pb.model.no_species):
            a, b = dev.download(0, "dens", s), port.dens(0, s)
            assert rel_err(a, b) <= 1e-12, (s, rel_err(a, b))
            dev.upload(0, "dens", b, s)
    dev.close()


def test_photo_refuses_trees(cuda_device):
    pb = workloads.amr(n_patches=6, levels=2, root_nr=32, root_nz=64, side_lo=8, side_hi=16, seed=1)
    t = CdrTree(pb.params, pb.model, pb.specs)
    with pytest.raises(Exception):
        t.set_photo(workloads.photo_model())
    t.close()


def test_photo_refuses_the_fused_entry_and_the_adjoint(cuda_device):
    """The fused two-launch step and the discrete adjoint carry no
    photoionization: with it on they refuse instead of dropping it."""
    import ctypes as C
    from arcos_b200.adjoint import Adjoint
    pb = workloads.photo(nr=16, nz=24, seed=2)
    dev = device_tree(pb, exact=False)
    assert dev.L.arcos_run_prepare(dev.h, C.c_double(50.0)) != 0
    with pytest.raises(Exception):
        Adjoint(dev).forward(2, 2, h=50.0)
    dev.close()
