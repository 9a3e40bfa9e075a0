"""The seeded workloads (CPU): the wavy field has the properties the parity
tests and the bench's wavy row rely on — both field components change sign
inside the kernels' 32-column / 16-row tiles, and |E| (with the applied
field added back) runs from below a reaction table's first node to above its
last — and the generators are deterministic in their seed."""
import numpy as np

from arcos_b200 import workloads


def _total_field(pb):
    er, ez, _ = pb.fields[0]
    return er + pb.params.E0_x, ez + pb.params.E0_z


def test_wavy_field_changes_sign_inside_tiles():
    pb = workloads.plain(nr=128, nz=256, field="wavy", seed=0)
    er, ez = _total_field(pb)
    er, ez = er[0, 2:-2, 2:-2], ez[0, 2:-2, 2:-2]      # interior (z rows, r columns)
    for comp in (er, ez):
        mixed = 0
        tiles = 0
        for z0 in range(0, comp.shape[0], 16):
            for c0 in range(0, comp.shape[1], 32):
                t = comp[z0:z0 + 16, c0:c0 + 32]
                tiles += 1
                mixed += bool((t > 0).any() and (t < 0).any())
        assert mixed >= tiles // 4, (mixed, tiles)


def test_wavy_field_sweeps_the_table():
    pb = workloads.plain(nr=128, nz=256, field="wavy", seed=0)
    er, ez = _total_field(pb)
    e = np.hypot(er[0, 2:-2, 2:-2], ez[0, 2:-2, 2:-2])
    table = pb.model.reactions[0].table          # nodes uniform in log10 |E| (reaction.c:127-136)
    lo, hi = 10.0 ** table.e_min, 10.0 ** (table.e_min + table.steps * table.e_step)
    assert e.min() < lo and e.max() > hi, (e.min(), e.max(), lo, hi)


def test_workloads_are_deterministic():
    a = workloads.plain(nr=32, nz=64, field="wavy", seed=3, noise=1e-3)
    b = workloads.plain(nr=32, nz=64, field="wavy", seed=3, noise=1e-3)
    c = workloads.plain(nr=32, nz=64, field="wavy", seed=4, noise=1e-3)
    for x, y in zip(a.fields[0][:2], b.fields[0][:2]):
        assert np.array_equal(x, y)
    assert np.array_equal(a.dens[0][0], b.dens[0][0])
    assert not np.array_equal(a.fields[0][0], c.fields[0][0])


def test_kinetic_wavy_full_sweeps_every_instance():
    pb = workloads.kinetic_batch(n_inst=3, points=300, sizes_r=(24, 40), sizes_z=(32, 48), seed=4,
                                 field="wavy_full")
    t = pb.model.reactions[0].table
    lo, hi = 10.0 ** t.e_min, 10.0 ** (t.e_min + t.steps * t.e_step)
    for f, E in zip(pb.fields, pb.family_E):
        er, ez, _ = f
        e = np.hypot(er[0, 2:-2, 2:-2] + E[0], ez[0, 2:-2, 2:-2] + E[2])
        assert (e < lo).any() and (e > hi).any(), (e.min(), e.max(), lo, hi)
    # the other field choices are unchanged by the option
    u = workloads.kinetic_batch(n_inst=3, points=300, sizes_r=(24, 40), sizes_z=(32, 48), seed=4,
                                field="wavy")
    assert u.family_E == pb.family_E and np.array_equal(u.dens[2][1], pb.dens[2][1])
