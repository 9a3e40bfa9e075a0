"""Refinement criteria on the device (arcos_cdr_refine) against the
reference's own cdr_refine (src/cdr.c:1630-1682, compiled into oracle/_ref)
on the same state: the child rectangles, their order and their
leading-edge flags must be identical.

Both sides refine the same arrays: the reference fills the density ghosts
(cdr_set_ext_bnd_r) and the charge (cdr_calc_charge_r); those arrays and a
seeded |E| field are then uploaded to the device unchanged, so the test
isolates the criteria, the maxima and the brick search."""
import numpy as np
import pytest

from arcos_b200 import workloads
from arcos_b200.cdr import CdrTree
from oracle import bind

pytestmark = pytest.mark.gpu

def seeded_state(pb, rng):
    """Two offset Gaussian blobs per species (ions shifted, so the charge has
    structure), a smooth |E| with a peak, on every grid of the tree."""
    out = []
    for sp in pb.specs:
        planes, nzt, nrt = sp.shape
        dr, dz = pb.params.dr(sp.level), pb.params.dz(sp.level)
        r = (np.arange(nrt) - 2 + sp.r0 + 0.5) * dr
        z = (np.arange(nzt) - 2 + sp.z0 + 0.5) * dz
        th = np.arange(planes)[:, None, None] * 0.3
        R, Z = np.meshgrid(r, z)
        Lz = pb.params.L_z
        per = []
        for s in range(pb.model.no_species):
            zc = Lz * (0.55 + 0.05 * s)
            blob = 0.1 * np.exp(-(R ** 2 + (Z - zc) ** 2) / (2 * (0.08 * Lz) ** 2))
            per.append((blob[None] * (1 + 0.1 * np.cos(th)) + 1e-6 * rng.random((planes, nzt, nrt))))
        eabs = (1.0 + 4.0 * np.exp(-(R ** 2 + (Z - 0.6 * Lz) ** 2) / (2 * (0.1 * Lz) ** 2)))[None] \
            * np.ones((planes, 1, 1))
        out.append((per, eabs))
    return out


def setup_pair(pb, seed=0):
    rng = np.random.default_rng(seed)
    st = seeded_state(pb, rng)
    ref = bind.RefTree(pb.params, pb.model, pb.specs, field_mode=bind.FIELD_FIXED)
    for g, (per, eabs) in enumerate(st):
        for s, a in enumerate(per):
            ref.dens(g, s)[...] = a
        ref.array(g, "eabs")[...] = eabs
    ref.call("ref_set_ext_bnd_r")
    ref.call("ref_calc_charge_r")
    dev = CdrTree(pb.params, pb.model, pb.specs)
    for g in range(len(pb.specs)):
        for s in range(pb.model.no_species):
            dev.upload(g, "dens", ref.dens(g, s).copy(), s)
        dev.upload(g, "charge", ref.array(g, "charge").copy())
        dev.upload(g, "eabs", ref.array(g, "eabs").copy())
    return ref, dev


CASES = [
    # threshold_eabs, level_eabs, threshold_charge, threshold_dens, threshold_edge, bdr, bdz, edge
    (1e9, 0, 1e9, 1e9, 1e9, 8, 8, False),
    (0.2, 4, 0.004, 0.004, 1e4, 8, 8, True),        # the reference's defaults (src/cstream.c:165-182)
    (1e9, 0, 1e9, 0.05, 1e9, 8, 8, False),
    (1e9, 0, 1e9, 0.01, 1e9, 8, 8, False),
    (1e9, 0, 1e9, 0.002, 1e9, 4, 16, False),
    (1e9, 0, 0.05, 1e9, 1e9, 8, 8, False),
    (1e9, 0, 0.005, 1e9, 1e9, 7, 5, False),
    (3.0, 3, 1e9, 1e9, 1e9, 8, 8, False),
    (1.5, 3, 1e9, 0.05, 1e9, 8, 8, False),
    (1e9, 0, 1e9, 0.05, 1e-2, 8, 8, True),
    (1e9, 0, 1e9, 0.01, 1e-4, 8, 8, True),
    (1e9, 0, 0.01, 0.02, 1e-3, 5, 7, True),
    (1e9, 0, 1e9, 0.01, 1e-4, 1, 2, True),          # one-cell bricks: the border recursion crosses bricks
    (1e9, 0, 0.02, 0.03, 1e9, 3, 1, False),
]


def run_cases(ref, dev, grids):
    results = []
    for case in CASES:
        te, le, tc, td, tg, bdr, bdz, edge = case
        for g in grids:
            a = ref.cdr_refine(g, te, le, tc, td, tg, bdr, bdz, 4, edge)
            b = dev.cdr_refine(g, te, le, tc, td, tg, bdr, bdz, 4, edge)
            assert a == b, (case, g, a, b)
            results.append(len(a))
    return results


@pytest.mark.parametrize("ion_mass", [0.0, 1.0])
def test_refine_2d_matches_reference(cuda_device, ion_mass):
    pb = workloads.plain(nr=48, nz=96, ion_mass=ion_mass, noise=0.0, seed=1)
    ref, dev = setup_pair(pb, seed=3)
    counts = run_cases(ref, dev, [0])
    # the cases span no refinement, partial refinement and refinement everywhere
    assert min(counts) == 0 and max(counts) > 2 and len(set(counts)) > 2
    dev.close()


def test_refine_3d_matches_reference(cuda_device):
    pb = workloads.plain(nr=40, nz=72, ntheta=4, ion_mass=1.0, noise=0.0, seed=2)
    ref, dev = setup_pair(pb, seed=4)
    counts = run_cases(ref, dev, [0])
    assert max(counts) > 0
    dev.close()


def test_refine_children_inherit_root_maxima(cuda_device):
    pb = workloads.amr(n_patches=8, levels=2, root_nr=32, root_nz=64, side_lo=8, side_hi=24, seed=5)
    ref, dev = setup_pair(pb, seed=6)
    kids = [g for g, sp in enumerate(pb.specs) if sp.parent == 0 and sp.nr >= 3 and sp.nz >= 3]
    assert kids
    run_cases(ref, dev, [0] + kids)
    dev.close()


def test_refine_rejects_narrow_grids_and_small_buffers(cuda_device):
    pb = workloads.plain(nr=48, nz=96, ion_mass=1.0, noise=0.0, seed=1)
    ref, dev = setup_pair(pb, seed=3)
    import ctypes as C
    from arcos_b200._lib import RefineParams
    rp = RefineParams(1e9, 0, 1e9, 1e-6, 1e9, 8, 8, 4)
    n = C.c_int(0)
    buf = (C.c_int * 5)()
    rc = dev.L.arcos_cdr_refine(dev.h, dev.ids[0], C.byref(rp), 0, buf, 1, C.byref(n))
    assert rc != 0 and n.value > 1
    assert len(dev.cdr_refine(0, 1e9, 0, 1e9, 1e-6, 1e9)) == n.value
    dev.close()
