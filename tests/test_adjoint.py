"""Discrete adjoint of the fused RK2 step against central finite differences
(step 1e-6 relative) of the forward map with the step sizes frozen to the
recorded sequence: the device forward, and at a smaller size the CPU oracle
(oracle/cdr_port.c, itself pinned to the reference sources).

The objective is J = 1/2 sum (n_e(T) - n_target)^2 * cell_volume with
cell_volume = 2 pi r_i dr dz; the parameters are the initial electron and
ion densities, the electron mobility 1/mass, diffusion_coeff and the alpha
table values.
"""
import copy

import numpy as np
import pytest

from arcos_b200 import workloads
from arcos_b200.adjoint import Adjoint, cell_volume, fd_objective_difference, smooth_direction
from arcos_b200.cdr import CdrTree
from oracle import bind
from parity_util import port_tree

pytestmark = pytest.mark.gpu

EPS = 1e-6
TOL = 1e-6


def problem(nr, nz, seed=0, ion_mass=0.0, field="uniform"):
    pb = workloads.plain(nr=nr, nz=nz, ion_mass=ion_mass, noise=1e-3, seed=seed, field=field)
    return pb


class Params:
    """The differentiated inputs: densities (interior), mobility, D, table."""

    def __init__(self, pb):
        self.dens = [a.copy() for a in pb.dens[0]]
        self.mu = np.array([1.0 / s.mass if s.mass > 0 else 0.0 for s in pb.model.species])
        self.D = pb.params.diffusion_coeff
        t = pb.model.reactions[0].table
        self.table = np.array(t.values[: t.steps + 1], dtype=np.float64)

    def perturbed(self, dirs, eps):
        q = copy.deepcopy(self)
        for s in range(len(q.dens)):
            q.dens[s][0, 2:-2, 2:-2] *= 1.0 + eps * dirs["dens"][s]
        q.mu = q.mu * (1.0 + eps * dirs["mu"])
        q.D = q.D * (1.0 + eps * dirs["D"])
        q.table = q.table * (1.0 + eps * dirs["table"])
        return q


def smooth_field(rng, nz, nr, modes=4):
    return smooth_direction(rng, nz, nr, modes)


def directions(pb, rng, which):
    spec = pb.specs[0]
    ns = pb.model.no_species
    z = {"dens": [np.zeros((spec.nz, spec.nr)) for _ in range(ns)], "mu": np.zeros(ns), "D": 0.0,
         "table": np.zeros(pb.model.reactions[0].table.steps + 1)}
    if "dens" in which:
        z["dens"] = [smooth_field(rng, spec.nz, spec.nr) for _ in range(ns)]
    if "mu" in which:
        z["mu"] = np.array([rng.standard_normal() if s.mass > 0 else 0.0 for s in pb.model.species])
    if "D" in which:
        z["D"] = rng.standard_normal()
    if "table" in which:
        z["table"] = rng.standard_normal(z["table"].shape)
    return z


def predicted(grads, base, dirs):
    """sum_i dJ/dx_i * x_i * d_i for the relative perturbation x_i (1 + eps d_i)."""
    v = 0.0
    for s in range(len(base.dens)):
        v += np.sum(grads.dens0[0][s][0, 2:-2, 2:-2] * base.dens[s][0, 2:-2, 2:-2] * dirs["dens"][s])
    v += np.sum(grads.mobility * base.mu * dirs["mu"])
    v += grads.diffusion * base.D * dirs["D"]
    v += np.sum(grads.tables[0] * base.table * dirs["table"])
    return v


def apply_device(tree, pb, q):
    for s, a in enumerate(q.dens):
        tree.upload(0, "dens", a, s)
    for s, sp in enumerate(pb.model.species):
        if sp.mass > 0:
            tree.set_species_mass(s, 1.0 / q.mu[s])
    tree.set_diffusion(q.D)
    t = pb.model.reactions[0].table
    tree.set_table_values(0, q.table, t.underflow, t.overflow)


def objective(ne, target, vol):
    return 0.5 * float(np.sum((ne - target) ** 2 * vol))


def device_setup(nr, nz, K, ck, seed=0, field="uniform"):
    pb = problem(nr, nz, seed=seed, field=field)
    tree = CdrTree(pb.params, pb.model, pb.specs)
    tree.set_fixed_field(pb.fields)
    adj = Adjoint(tree)
    base = Params(pb)
    apply_device(tree, pb, base)
    # target: forward run from a perturbed seed (amplitude x1.1, radius x0.9)
    spec = pb.specs[0]
    rng = np.random.default_rng(seed + 100)
    tgt_e = workloads.seed_dens(spec, pb.params, rng, amp=0.11, sigma=0.09, noise=1e-3)
    tree.upload(0, "dens", tgt_e, 0)
    tree.upload(0, "dens", tgt_e, 1)
    tree.run(K, 50.0)
    target = tree.download(0, "dens", 0)
    apply_device(tree, pb, base)
    hs = adj.forward(K, ck, h=50.0)
    vol = cell_volume(spec, pb.params.dr(0), pb.params.dz(0))
    return pb, tree, adj, base, hs, target, vol


def device_grads(tree, adj, target, vol):
    ne = tree.download(0, "dens", 0)
    lam = (ne - target) * vol
    adj.set_cotangent(0, 0, lam)
    adj.set_cotangent(0, 1, np.zeros_like(lam))
    return adj.backward(), objective(ne, target, vol)


def device_ne(tree, adj, pb, q, hs, K, ck):
    apply_device(tree, pb, q)
    adj.forward(K, ck, h_seq=hs)
    return tree.download(0, "dens", 0)


def fd_difference(ne_p, ne_m, target, vol, eps):
    return fd_objective_difference(ne_p, ne_m, target, vol, eps)


def device_J(tree, adj, pb, q, hs, K, ck, target, vol):
    return objective(device_ne(tree, adj, pb, q, hs, K, ck), target, vol)


@pytest.mark.parametrize("ck", [4, 16])
@pytest.mark.parametrize("field", ["uniform", "wavy"])
@pytest.mark.parametrize("which", [("dens",), ("mu",), ("D",), ("table",), ("dens", "mu", "D", "table")])
def test_adjoint_matches_device_fd(cuda_device, which, field, ck):
    """Uniform applied field, and the non-uniform wavy field (radial drift,
    sign changes of the velocity inside a warp, |E| over the whole table);
    checkpoints every 4 steps (segments recomputed), or one segment (every
    state kept by the forward run)."""
    K = 16
    pb, tree, adj, base, hs, target, vol = device_setup(32, 64, K, ck, seed=1, field=field)
    grads, J0 = device_grads(tree, adj, target, vol)
    assert J0 > 0
    rng = np.random.default_rng(7)
    # A table-only direction moves n_e(T) by ~1e-11 relative at this size, so a
    # 1e-6 step leaves the difference of the two runs at rounding level; the
    # rate is linear in the table values, so a 1e-4 step has no truncation
    # error to speak of.  Every other direction uses the 1e-6 step.
    eps = 1e-4 if which == ("table",) else EPS
    for _ in range(2):
        dirs = directions(pb, rng, which)
        ne_p = device_ne(tree, adj, pb, base.perturbed(dirs, eps), hs, K, ck)
        ne_m = device_ne(tree, adj, pb, base.perturbed(dirs, -eps), hs, K, ck)
        fd = fd_difference(ne_p, ne_m, target, vol, eps)
        pr = predicted(grads, base, dirs)
        assert abs(fd - pr) <= TOL * max(abs(fd), 1e-300), (which, fd, pr)


@pytest.mark.parametrize("field", ["uniform", "wavy"])
def test_adjoint_matches_oracle_fd(cuda_device, field):
    """FD of the CPU oracle's frozen-step forward against the device adjoint."""
    K, ck, nr, nz = 8, 4, 24, 48
    pb, tree, adj, base, hs, target, vol = device_setup(nr, nz, K, ck, seed=2, field=field)
    grads, _ = device_grads(tree, adj, target, vol)

    def oracle_ne(q):
        pq = copy.deepcopy(pb)
        pq.dens = [[a.copy() for a in q.dens]]
        for s, sp in enumerate(pq.model.species):
            if sp.mass > 0:
                sp.mass = 1.0 / q.mu[s]
        pq.params.diffusion_coeff = q.D
        pq.model.reactions[0].table.values = q.table.copy()
        port = port_tree(pq)
        for k in range(K):
            port.rk2_frozen(float(hs[0, k]))
        return port.dens(0, 0).copy()

    rng = np.random.default_rng(11)
    for _ in range(2):
        dirs = directions(pb, rng, ("dens", "mu", "D", "table"))
        fd = fd_difference(oracle_ne(base.perturbed(dirs, EPS)), oracle_ne(base.perturbed(dirs, -EPS)),
                           target, vol, EPS)
        pr = predicted(grads, base, dirs)
        assert abs(fd - pr) <= TOL * abs(fd), (fd, pr)


@pytest.mark.parametrize("ck", [4, 6])
def test_adjoint_keeps_forward_state(cuda_device, ck):
    K = 6
    pb, tree, adj, base, hs, target, vol = device_setup(32, 64, K, ck, seed=3)
    before = [tree.download(0, "dens", s) for s in range(2)]
    device_grads(tree, adj, target, vol)
    for s in range(2):
        assert np.array_equal(tree.download(0, "dens", s)[0, 2:-2, 2:-2], before[s][0, 2:-2, 2:-2])


@pytest.mark.parametrize("ck", [4, 10])
def test_frozen_forward_reproduces_cfl_run(cuda_device, ck):
    """The frozen-step forward with the recorded sizes gives the CFL run's state."""
    K = 10
    pb, tree, adj, base, hs, target, vol = device_setup(32, 64, K, ck, seed=4)
    a = [tree.download(0, "dens", s) for s in range(2)]
    apply_device(tree, pb, base)
    adj.forward(K, ck, h_seq=hs)
    for s in range(2):
        assert np.array_equal(tree.download(0, "dens", s)[0, 2:-2, 2:-2], a[s][0, 2:-2, 2:-2])


def test_kept_states_give_the_checkpointed_gradients(cuda_device):
    """One segment (states kept by the forward run) and checkpoints every 3
    steps (segments recomputed with the recorded step sizes) give the same
    gradients: the recomputed states are the forward's, bit for bit, so the
    density, mobility and diffusion gradients are identical (the table
    gradients to the order of their atomic sums)."""
    K = 9
    out = []
    for ck in (3, 9):
        pb, tree, adj, base, hs, target, vol = device_setup(32, 64, K, ck, seed=6, field="wavy")
        g, _ = device_grads(tree, adj, target, vol)
        out.append((g, hs))
        tree.close()
    (ga, ha), (gb, hb) = out
    assert np.array_equal(ha, hb)
    for s in range(2):
        assert np.array_equal(ga.dens0[0][s], gb.dens0[0][s]), s
    assert np.array_equal(ga.mobility, gb.mobility) and ga.diffusion == gb.diffusion
    # the table gradients are sums of atomic additions, whose order varies
    ta, tb = ga.tables[0], gb.tables[0]
    assert np.max(np.abs(ta - tb)) <= 1e-12 * np.max(np.abs(tb))


@pytest.mark.parametrize("field,ck", [("uniform", 3), ("wavy", 6)])
def test_kinetic_batch_adjoint_matches_fd(cuda_device, field, ck):
    """Three families of different sizes, six species (ions mobile), nine
    reactions with one- and two-input terms: the adjoint of the total electron
    number at T with respect to the initial densities of every species and
    every table value, against central differences of the frozen-step
    forward.  Two checkpoint segments, or one (every state kept)."""
    pb = workloads.kinetic_batch(n_inst=3, points=200, sizes_r=(24, 40), sizes_z=(32, 48), seed=1,
                                 field=field)
    ns = pb.model.no_species
    tree = CdrTree(pb.params, pb.model, pb.specs)
    for f, E in enumerate(pb.family_E):
        tree.set_family_field(f, *E)
    tree.set_fixed_field(pb.fields)
    tabs = [np.array(r.table.values[: r.table.steps + 1], dtype=np.float64) for r in pb.model.reactions]

    def apply(dens, vals):
        for g, per in enumerate(dens):
            for s, a in enumerate(per):
                tree.upload(g, "dens", a, s)
        for r, re in enumerate(pb.model.reactions):
            tree.set_table_values(r, vals[r], re.table.underflow, re.table.overflow)

    K = 6
    adj = Adjoint(tree)
    apply(pb.dens, tabs)
    hs = adj.forward(K, ck, h=50.0)
    vols = [cell_volume(sp, pb.params.dr(0), pb.params.dz(0)) for sp in pb.specs]
    for g, sp in enumerate(pb.specs):
        adj.set_cotangent(g, 0, vols[g])
        for s in range(1, ns):
            adj.set_cotangent(g, s, np.zeros(sp.shape))
    grads = adj.backward()

    def total_electrons(dens, vals):
        apply(dens, vals)
        adj.forward(K, ck, h_seq=hs)
        return [tree.download(g, "dens", 0) for g in range(len(pb.specs))]

    rng = np.random.default_rng(23)
    for which, eps in ((("dens", "table"), EPS), (("table",), 1e-4)):
        dd = []
        for g, sp in enumerate(pb.specs):
            per = []
            for s in range(ns):
                d = np.zeros(sp.shape)
                if "dens" in which:
                    d[0, 2:-2, 2:-2] = smooth_direction(rng, sp.nz, sp.nr)
                per.append(d)
            dd.append(per)
        dv = [rng.standard_normal(t.shape) if "table" in which else np.zeros(t.shape) for t in tabs]
        pred = sum(float(np.sum(grads.dens0[g][s] * pb.dens[g][s] * dd[g][s]))
                   for g in range(len(pb.specs)) for s in range(ns))
        pred += sum(float(np.sum(grads.tables[r] * tabs[r] * dv[r])) for r in range(len(tabs)))
        outs = []
        for sg in (1.0, -1.0):
            dens = [[pb.dens[g][s] * (1.0 + sg * eps * dd[g][s]) for s in range(ns)] for g in range(len(pb.specs))]
            vals = [tabs[r] * (1.0 + sg * eps * dv[r]) for r in range(len(tabs))]
            outs.append(total_electrons(dens, vals))
        fd = sum(float(np.sum(vols[g] * (outs[0][g] - outs[1][g]))) for g in range(len(pb.specs))) / (2 * eps)
        assert abs(fd - pred) <= TOL * abs(fd), (which, fd, pred)
    tree.close()


def test_vjp_forms_give_the_same_gradients(cuda_device):
    """The transposed step as one kernel and as faces + reactions (the
    automatic choice from four species on): the density gradients bit for
    bit (every value computed with the same operations in the same order),
    the mobility, diffusion and table sums to the order of their partial
    sums."""
    pb = workloads.kinetic_batch(n_inst=3, points=200, sizes_r=(24, 40), sizes_z=(32, 48), seed=4,
                                 field="wavy")
    ns = pb.model.no_species
    out = []
    for form in (0, 1):
        tree = CdrTree(pb.params, pb.model, pb.specs)
        for f, E in enumerate(pb.family_E):
            tree.set_family_field(f, *E)
        tree.set_fixed_field(pb.fields)
        for g, per in enumerate(pb.dens):
            for s, a in enumerate(per):
                tree.upload(g, "dens", a, s)
        assert tree.L.arcos_set_vjp_form(tree.h, form) == 0
        adj = Adjoint(tree)
        adj.forward(5, 5, h=50.0)
        for g, sp in enumerate(pb.specs):
            for s in range(ns):
                adj.set_cotangent(g, s, cell_volume(sp, pb.params.dr(0), pb.params.dz(0)) * (1.0 + 0.1 * s))
        out.append(adj.backward())
        tree.close()
    a, b = out
    for g in range(len(pb.specs)):
        for s in range(ns):
            assert np.array_equal(a.dens0[g][s], b.dens0[g][s]), (g, s)
    assert np.allclose(a.mobility, b.mobility, rtol=1e-12, atol=0)
    assert abs(a.diffusion - b.diffusion) <= 1e-12 * abs(b.diffusion)
    for r in range(len(a.tables)):
        ta, tb = a.tables[r], b.tables[r]
        assert np.max(np.abs(ta - tb)) <= 1e-12 * max(np.max(np.abs(tb)), 1e-300), r
