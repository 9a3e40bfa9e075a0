"""Host-side logic without a GPU: reaction-table files, grid geometry, the
synthetic workloads of the benchmark configurations, FD helpers."""
import numpy as np
import pytest

from arcos_b200 import workloads
from arcos_b200.adjoint import cell_volume, fd_objective_difference, smooth_direction
from arcos_b200.grids import GridSpec, inherit_ext_bound
from arcos_b200.model import BND_MASK_ALL, BND_MASK_BOTTOM, BND_MASK_LEFT, minimal_model
from arcos_b200.react_table import log_uniform_table, react_table_read, write_react_table


def test_react_table_roundtrip_is_bit_exact(tmp_path):
    t = log_uniform_table(lambda e: e * np.exp(-1.0 / e), 0.05, 20.0, 256)
    p = tmp_path / "alpha.reaction"
    write_react_table(p, t, "minimal model")
    u = react_table_read(p)
    assert (u.e_min, u.e_step, u.steps, u.underflow, u.overflow) == \
        (t.e_min, t.e_step, t.steps, t.underflow, t.overflow)
    assert np.array_equal(u.values, t.values)
    assert len(t.padded_values()) == t.steps + 2


def test_grid_shapes_and_interior():
    g2 = GridSpec(0, 0, 8, 12)
    assert g2.shape == (1, 16, 12) and g2.planes == 1 and g2.theta0 == 0
    g3 = GridSpec(0, 0, 8, 12, ntheta=4)
    assert g3.shape == (8, 16, 12) and g3.theta0 == -2
    a = g3.zeros()
    g3.interior(a)[...] = 1.0
    assert a.sum() == 4 * 12 * 8


def test_inherit_ext_bound():
    parent = GridSpec(0, 0, 16, 16, ext_bound=BND_MASK_ALL)
    child = GridSpec(0, 0, 8, 8, level=1)          # left and bottom edges shared
    assert inherit_ext_bound(parent, child) == BND_MASK_LEFT | BND_MASK_BOTTOM


def test_amr_workload_has_the_configured_tree():
    pb = workloads.amr()
    assert len(pb.specs) == 320
    levels = [sp.level for sp in pb.specs]
    assert sorted(set(levels)) == [0, 1, 2, 3]
    for sp in pb.specs[1:]:
        p = pb.specs[sp.parent]
        assert p.level == sp.level - 1
        assert 2 * p.r0 <= sp.r0 and sp.r1 <= 2 * p.r1 and 2 * p.z0 <= sp.z0 and sp.z1 <= 2 * p.z1


def test_kinetic_batch_shapes():
    pb = workloads.kinetic_batch(n_inst=5, points=50)
    assert len(pb.specs) == 5 and len(pb.family_E) == 5
    assert pb.model.no_species == 6 and len(pb.model.reactions) == 9
    for sp in pb.specs:
        assert sp.nr in (64, 128, 256) and sp.nz in (128, 256, 512)
    assert all(-2.0 <= E[2] <= -0.5 for E in pb.family_E)


def test_minimal_model_table():
    m = minimal_model(ion_mass=0.0, points=256)
    t = m.reactions[0].table
    assert t.steps == 255 and m.species[1].mass == 0.0
    assert t.values[0] == pytest.approx(0.05 * np.exp(-20.0))


def test_fd_helpers():
    spec = GridSpec(0, 0, 4, 3)
    v = cell_volume(spec, 0.5, 0.25)
    assert v[0, 2, 2] == pytest.approx(2 * np.pi * 0.25 * 0.5 * 0.25) and v[0, 0, 0] == 0
    rng = np.random.default_rng(0)
    d = smooth_direction(rng, 16, 8)
    assert d.shape == (16, 8) and np.all(np.isfinite(d))
    a, b, t = np.full(3, 2.0), np.full(3, 1.0), np.zeros(3)
    vol = np.ones(3)
    # J = 1/2 sum n^2: (J(2) - J(1)) / (2 * 0.5) = 3 * 1.5 / 1
    assert fd_objective_difference(a, b, t, vol, 0.5) == pytest.approx(4.5)
