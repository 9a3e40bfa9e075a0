"""Device against the CPU oracle at the sizes of the five benchmark
configurations (seeded synthetic inputs of the configured shapes):

* c0: 128 x 256, 2 species (immobile ions), field solve in the loop (the
  host Poisson stand-in at the pois_solve_a seam, on both sides), 200 RK2
  steps compared after every step;
* c1: 512 x 1024 cells x 16 theta planes, fixed field, drift/diffusion on
  every plane (the benchmark's default path), 2 steps;
* c2: the 320-patch, 4-level refinement tree, 2 steps of the batched step;
* c3: the adjoint's 256 x 512 grid, 64 steps with checkpoints every 8,
  against central finite differences of the device forward;
* c4: 32 uneven instances, 6 species, 9 reactions with 1000-point tables
  (the oracle pinned to a reference build with a 1024-entry table bound),
  2 steps.

Tolerance: 1e-12 relative per step (the state is resynchronised to the
oracle after each compared step where the kernel is the division-free one),
dt sequences equal to 1e-12.
"""
import numpy as np
import pytest

from arcos_b200 import workloads
from arcos_b200.adjoint import Adjoint, cell_volume, smooth_direction
from arcos_b200.cdr import CdrTree
from oracle import bind
from parity_util import port_tree, rel_err, single_family
from test_gpu_parity import device_tree

pytestmark = pytest.mark.gpu

TOL = 1e-12


def test_c0_field_in_loop_200_steps(cuda_device):
    pb = workloads.plain(nr=128, nz=256, ion_mass=0.0, seed=0)
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
    worst = 0.0
    for k in range(200):
        hp = port.rk2(50.0)[0]
        hd = dev.run(1, 50.0)[0][0]
        assert abs(hd - hp) <= TOL * hp, (k, hd, hp)
        for s in range(2):
            e = rel_err(dev.download(0, "dens", s), port.dens(0, s))
            worst = max(worst, e)
            assert e <= TOL, (k, s, e)
    dev.close()


def test_c1_full_grid_two_steps(cuda_device):
    pb = workloads.plain(nr=512, nz=1024, ntheta=16, ion_mass=1.0, noise=1e-6, seed=0)
    port = port_tree(pb, per_plane=True)
    dev = device_tree(pb, exact=False)
    for _ in range(2):
        hp = port.rk2(50.0)[0]
        hd = dev.run(1, 50.0)[0][0]
        assert abs(hd - hp) <= TOL * hp
        for s in range(2):
            a, b = dev.download(0, "dens", s), port.dens(0, s)
            assert rel_err(a, b) <= TOL, (s, rel_err(a, b))
            dev.upload(0, "dens", b, s)
    dev.close()


def test_c2_320_patch_tree_two_steps(cuda_device):
    pb = workloads.amr(seed=0)
    assert len(pb.specs) == 320 and max(s.level for s in pb.specs) == 3
    port = port_tree(pb, zero_all=True)
    dev = device_tree(pb, exact=False)
    for _ in range(2):
        hp = port.rk2(50.0)[0]
        hd = dev.run(1, 50.0)[0][0]
        assert abs(hd - hp) <= TOL * hp
        for g in range(len(pb.specs)):
            for s in range(2):
                a, b = dev.download(g, "dens", s), port.dens(g, s)
                assert rel_err(a, b) <= TOL, (g, s, rel_err(a, b))
                dev.upload(g, "dens", b, s)
    dev.close()


def test_c3_adjoint_full_size_fd(cuda_device):
    """256 x 512, K = 64 steps, checkpoints every 8: gradients of
    J = 1/2 sum (n_e(T) - n_target)^2 cell_volume with respect to the
    initial densities against central differences (step 1e-6 relative)."""
    K, ck = 64, 8
    pb = workloads.plain(nr=256, nz=512, ion_mass=0.0, noise=1e-3, seed=0)
    tree = CdrTree(pb.params, pb.model, pb.specs)
    tree.set_fixed_field(pb.fields)
    adj = Adjoint(tree)
    spec = pb.specs[0]
    rng = np.random.default_rng(100)
    tgt = workloads.seed_dens(spec, pb.params, rng, amp=0.11, sigma=0.09, noise=1e-3)
    for s in range(2):
        tree.upload(0, "dens", tgt, s)
    tree.run(K, 50.0)
    target = tree.download(0, "dens", 0)
    for s in range(2):
        tree.upload(0, "dens", pb.dens[0][s], s)
    hs = adj.forward(K, ck, h=50.0)
    vol = cell_volume(spec, pb.params.dr(0), pb.params.dz(0))
    ne = tree.download(0, "dens", 0)
    adj.set_cotangent(0, 0, (ne - target) * vol)
    adj.set_cotangent(0, 1, np.zeros_like(ne))
    g = adj.backward()

    def J(dens):
        for s in range(2):
            tree.upload(0, "dens", dens[s], s)
        adj.forward(K, ck, h_seq=hs)
        return tree.download(0, "dens", 0)

    for _ in range(3):
        d = [np.zeros(spec.shape) for _ in range(2)]
        for s in range(2):
            d[s][0, 2:-2, 2:-2] = smooth_direction(rng, spec.nz, spec.nr)
        eps = 1e-6
        plus = J([pb.dens[0][s] * (1 + eps * d[s]) for s in range(2)])
        minus = J([pb.dens[0][s] * (1 - eps * d[s]) for s in range(2)])
        fd = float(np.sum(((plus - target) ** 2 - (minus - target) ** 2) * vol)) * 0.25 / eps
        pred = sum(float(np.sum(g.dens0[0][s] * pb.dens[0][s] * d[s])) for s in range(2))
        assert abs(fd - pred) <= 1e-6 * abs(fd), (fd, pred)
    tree.close()


def test_c4_kinetic_batch_1000_point_tables(cuda_device):
    pb = workloads.kinetic_batch(seed=0)            # 32 instances, 1000-point tables
    assert len(pb.specs) == 32 and pb.model.reactions[0].table.points == 1000
    dev = device_tree(pb, exact=False)
    ports = [port_tree(single_family(pb, i), E=pb.family_E[i]) for i in range(32)]
    for _ in range(2):
        hd = dev.run(1, 50.0)
        for i, port in enumerate(ports):
            hp = port.rk2(50.0)[0]
            assert abs(hd[i][0] - hp) <= TOL * hp, (i, hd[i][0], hp)
            for s in range(6):
                a, b = dev.download(i, "dens", s), port.dens(0, s)
                assert rel_err(a, b) <= TOL, (i, s, rel_err(a, b))
                dev.upload(i, "dens", b, s)
    dev.close()
