"""Pins the CPU oracle (oracle/cdr_port.c) to the reference itself: the
reference C sources compiled from the reference tree (oracle/_ref), driven
through the same seeded inputs.  Only the Fortran drift/diffusion kernel is
not the reference's own binary code (no Fortran compiler here); it is the
literal array-at-a-time restatement of oracle/f90_restated.c, while the
oracle computes the same fluxes face by face, so agreement also checks that
reformulation.  Everything else on the path is the reference's C.

Skipped where the reference tree is absent (the build needs its sources).
"""
import numpy as np
import pytest

from arcos_b200 import workloads
from arcos_b200.grids import GridSpec
from arcos_b200.model import KineticModel, Params, Reaction, Species
from arcos_b200.react_table import ReactTable
from oracle import bind
from parity_util import max_ulp, port_tree, single_family

needs_ref = pytest.mark.skipif(not bind.ref_available(), reason="reference build absent")


def ref_tree(pb, field_mode=bind.FIELD_FIXED, E=None, variant="plain"):
    import copy
    params = copy.deepcopy(pb.params)
    if E is not None:
        params.E0_x, params.E0_y, params.E0_z = E
    t = bind.RefTree(params, pb.model, pb.specs, field_mode=field_mode, omp=variant)
    for g, per in enumerate(pb.dens):
        for s, a in enumerate(per):
            t.dens(g, s)[...] = a
    if field_mode == bind.FIELD_FIXED:
        for g, (er, ez, et) in enumerate(pb.fields):
            t.set_fixed_field(g, er, ez, et if et is not None else pb.specs[g].zeros())
    return t


def assert_same(port, ref, pb, what=("dens",)):
    for g in range(len(pb.specs)):
        for w in what:
            for s in range(pb.model.no_species):
                a, b = port.array(g, w, s), ref.array(g, w, s)
                assert max_ulp(a, b) == 0, (g, w, s, max_ulp(a, b))


@needs_ref
@pytest.mark.parametrize("ion_mass", [0.0, 1.0])
def test_plain_2d(ion_mass):
    pb = workloads.plain(nr=40, nz=80, ion_mass=ion_mass, noise=1e-3, seed=1)
    port, ref = port_tree(pb), ref_tree(pb)
    for _ in range(5):
        hp, st = port.rk2(50.0)
        hr = ref.rk2(50.0)
        assert st == 0 and hp == hr
    assert_same(port, ref, pb, ("dens", "d_dens"))


@needs_ref
def test_dirichlet_boundaries():
    pb = workloads.plain(nr=33, nz=47, ion_mass=1.0, noise=1e-3, seed=2)
    pb.params.cdr_bnd_top = -1
    pb.params.cdr_bnd_right = -1
    pb.params.cdr_bnd_bottom = -1
    port, ref = port_tree(pb), ref_tree(pb)
    for _ in range(4):
        assert port.rk2(50.0)[0] == ref.rk2(50.0)
    assert_same(port, ref, pb)


@needs_ref
def test_theta_ref_exact():
    """ntheta > 1 with the reference's literal behaviour: the Fortran gets the
    theta = -2 plane only, so the real planes see reactions only."""
    pb = workloads.plain(nr=20, nz=36, ntheta=4, ion_mass=1.0, noise=1e-6, seed=3)
    pb.params.per_plane = False
    port, ref = port_tree(pb, per_plane=False), ref_tree(pb)
    for _ in range(3):
        assert port.rk2(50.0)[0] == ref.rk2(50.0)
    assert_same(port, ref, pb, ("dens", "d_dens"))


@needs_ref
def test_theta_per_plane():
    pb = workloads.plain(nr=20, nz=36, ntheta=4, ion_mass=1.0, noise=1e-6, seed=4)
    port, ref = port_tree(pb, per_plane=True), ref_tree(pb)
    for _ in range(3):
        assert port.rk2(50.0)[0] == ref.rk2_sw(50.0, per_plane=True, zero_all=False)
    assert_same(port, ref, pb, ("dens", "d_dens"))


@needs_ref
def test_amr_tree():
    pb = workloads.amr(n_patches=14, levels=3, root_nr=32, root_nz=64, side_lo=8, side_hi=24, seed=5)
    port, ref = port_tree(pb, zero_all=True), ref_tree(pb)
    for _ in range(3):
        assert port.rk2(50.0)[0] == ref.rk2_sw(50.0, per_plane=False, zero_all=True)
    assert_same(port, ref, pb)


@needs_ref
def test_amr_deep():
    pb = workloads.amr(n_patches=20, levels=4, root_nr=32, root_nz=64, side_lo=8, side_hi=32, seed=6)
    port, ref = port_tree(pb, zero_all=True), ref_tree(pb)
    for _ in range(2):
        assert port.rk2(50.0)[0] == ref.rk2_sw(50.0, per_plane=False, zero_all=True)
    assert_same(port, ref, pb)


@needs_ref
def test_field_in_loop():
    pb = workloads.plain(nr=24, nz=48, ion_mass=0.0, seed=7)
    port = port_tree(pb, field_mode=bind.FIELD_POISSON)
    ref = ref_tree(pb, field_mode=bind.FIELD_POISSON)
    port.call("port_calc_charge")
    ref.call("ref_calc_charge_r")
    for _ in range(3):
        assert port.rk2(50.0)[0] == ref.rk2(50.0)
    assert_same(port, ref, pb, ("dens", "er", "ez", "eabs"))


@needs_ref
def test_kinetic_model():
    pb = workloads.kinetic_batch(n_inst=2, points=300, sizes_r=(24,), sizes_z=(40,), seed=8)
    for i in range(2):
        sub = single_family(pb, i)
        port = port_tree(sub, E=pb.family_E[i])
        ref = ref_tree(sub, E=pb.family_E[i])
        for _ in range(3):
            assert port.rk2(50.0)[0] == ref.rk2(50.0)
        assert_same(port, ref, sub, ("dens", "d_dens"))


@needs_ref
@pytest.mark.parametrize("ion_mass", [0.0, 1.0])
def test_plain_2d_wavy_field(ion_mass):
    """Non-uniform field (both components change sign, |E| from table
    underflow to overflow): radial drift and the lookup at every node."""
    pb = workloads.plain(nr=40, nz=72, ion_mass=ion_mass, noise=1e-3, seed=13, field="wavy")
    port, ref = port_tree(pb), ref_tree(pb)
    for _ in range(5):
        hp, st = port.rk2(50.0)
        assert st == 0 and hp == ref.rk2(50.0)
    assert_same(port, ref, pb, ("dens", "d_dens"))


@needs_ref
def test_theta_ref_exact_wavy_field():
    pb = workloads.plain(nr=20, nz=36, ntheta=4, ion_mass=1.0, noise=1e-6, seed=3, field="wavy")
    pb.params.per_plane = False
    port, ref = port_tree(pb, per_plane=False), ref_tree(pb)
    for _ in range(3):
        assert port.rk2(50.0)[0] == ref.rk2(50.0)
    assert_same(port, ref, pb, ("dens", "d_dens"))


@needs_ref
@pytest.mark.parametrize("field", ["wavy", "wavy_full"])
def test_kinetic_model_wavy_field(field):
    """Nine reactions on a non-uniform field: "wavy" keeps |E| near each
    instance's applied field (a few table nodes), "wavy_full" sweeps it from
    below the tables' first node to above their last."""
    pb = workloads.kinetic_batch(n_inst=2, points=300, sizes_r=(24,), sizes_z=(40,), seed=8,
                                 field=field)
    for i in range(2):
        sub = single_family(pb, i)
        port = port_tree(sub, E=pb.family_E[i])
        ref = ref_tree(sub, E=pb.family_E[i])
        for _ in range(3):
            assert port.rk2(50.0)[0] == ref.rk2(50.0)
        assert_same(port, ref, sub, ("dens", "d_dens"))


@pytest.mark.skipif(not bind.ref_available("bigtab"), reason="reference build absent")
@pytest.mark.parametrize("field", ["uniform", "wavy", "wavy_full"])
def test_kinetic_model_1000_point_tables(field):
    """The kinetic batch's 1000-point tables, against the reference built
    with a 1024-entry MAX_TABLE_SIZE (oracle/react_table_1024.h): 9
    reactions, 6 species; with "wavy_full" |E| runs over the whole table
    and beyond both of its ends."""
    pb = workloads.kinetic_batch(n_inst=2, points=1000, sizes_r=(24,), sizes_z=(40,), seed=8,
                                 field=field)
    for i in range(2):
        sub = single_family(pb, i)
        port = port_tree(sub, E=pb.family_E[i])
        ref = ref_tree(sub, E=pb.family_E[i], variant="bigtab")
        for _ in range(3):
            assert port.rk2(50.0)[0] == ref.rk2(50.0)
        assert_same(port, ref, sub, ("dens", "d_dens"))


def test_plain_reference_refuses_tables_above_500_points():
    pb = workloads.kinetic_batch(n_inst=1, points=1000, sizes_r=(24,), sizes_z=(40,), seed=8)
    if not bind.ref_available("plain"):
        pytest.skip("reference build absent")
    with pytest.raises(ValueError, match="500"):
        ref_tree(single_family(pb, 0), E=pb.family_E[0])


@needs_ref
def test_courant_and_pieces():
    pb = workloads.plain(nr=24, nz=40, ion_mass=1.0, noise=1e-3, seed=9)
    port, ref = port_tree(pb), ref_tree(pb)
    port.calc_field()
    ref.call("ref_calc_field")
    assert port.courant()[0] == ref.courant()
    port.call("port_calc_d_dens_grid")
    ref.call("ref_calc_d_dens")
    assert_same(port, ref, pb, ("d_dens", "eabs", "er", "ez"))


@needs_ref
def test_narrow_seam_limiter_branches():
    """The per-face flux against the literal Fortran restatement on random
    slabs that hit every limiter branch, both velocity signs and the
    |dC| <= 1e-20 mask."""
    rng = np.random.default_rng(10)
    ref = bind.ref_lib()
    port = bind.port_lib()
    P = bind._dp
    for trial in range(20):
        r0 = int(rng.integers(0, 6))
        z0 = int(rng.integers(0, 4))
        r1, z1 = r0 + int(rng.integers(2, 20)), z0 + int(rng.integers(2, 20))
        shape = (z1 - z0 + 4, r1 - r0 + 4)
        dens = rng.random(shape) ** 3
        if trial % 3 == 0:
            dens[:, : shape[1] // 2] = 0.25           # flat region: |dC| == 0
        if trial % 4 == 1:
            dens = np.cumsum(rng.random(shape), axis=1)   # monotone: p in (0, 4)
        er = rng.normal(size=shape)
        ez = rng.normal(size=shape)
        er[er > 1.0] = 0.0                               # v == 0 faces
        d0 = rng.normal(size=shape)
        a, b = d0.copy(), d0.copy()
        mass = float(rng.choice([1.0, 0.5, 100.0]))
        charge = float(rng.choice([-1.0, 1.0]))
        ref.ref_advect_vec(mass, charge, P(dens), P(a), P(er), er.size, P(ez), ez.size, 0.1,
                           1 / 64, 1 / 32, r0, r1, z0, z1)
        port.port_advect_vec(mass, charge, P(dens), P(b), P(er), P(ez), 0.1, 1 / 64, 1 / 32,
                             r0, r1, z0, z1)
        assert max_ulp(a, b) == 0, trial


def _kat_problem(table: ReactTable, evals):
    """One immobile charged species with a source reaction (no inputs) whose
    rate is the table lookup; the field is set so |E| of column i is evals[i]."""
    nr = len(evals)
    params = Params(L_r=1.0, L_z=1.0, gridpoints_r=nr, gridpoints_z=4, E0_z=0.0,
                    warn_min_timestep=0.0, max_levels=2)
    model = KineticModel([Species("x", 1.0, 0.0)], [Reaction([], [0], table)])
    spec = GridSpec(0, 0, nr, 4)
    ez = spec.zeros()
    ez[0, :, 2:nr + 2] = np.asarray(evals)[None, :]
    return workloads.Problem(params, model, [spec], [[spec.zeros() + 1.0]],
                             [(spec.zeros(), ez, None)])


def test_table_known_answer():
    """The worked example of react_table.c:41-62: k(E) = E on 4 nodes
    E = 10^{-2..1}; inside the range the lookup returns E (to rounding),
    below it the underflow value 0, above it the overflow value 100."""
    import os
    import tempfile
    from arcos_b200.react_table import react_table_read
    text = ("Sample reaction table. k(E) = E. 4 points are defined at E = 10^i, i in {-2,-1,0,1}.\n"
            "START\n-2.0\n1\n4\n0.0\n100.0\n0.01\n0.1\n1.0\n10.0\nThis bit is ignored.\n")
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "kat.reaction")
        with open(path, "w") as fp:
            fp.write(text)
        table = react_table_read(path)
    assert (table.e_min, table.e_step, table.steps) == (-2.0, 1.0, 3)
    evals = [0.005, 0.011, 0.05, 0.3, 2.0, 9.5, 12.0, 1000.0]
    pb = _kat_problem(table, evals)
    port = port_tree(pb)
    port.calc_field()
    port.call("port_calc_d_dens_grid")
    got = port.array(0, "d_dens", 0)[0, 3, 2:2 + len(evals)]
    expect = [0.0 if e < 0.01 else (100.0 if e > 10.0 else e) for e in evals]
    assert np.allclose(got, expect, rtol=1e-14, atol=0)
    if bind.ref_available():
        ref = ref_tree(pb)
        ref.call("ref_calc_field")
        ref.call("ref_calc_d_dens")
        assert max_ulp(ref.array(0, "d_dens", 0), port.array(0, "d_dens", 0)) == 0


def test_uniform_density_zero_flux():
    """No radial field and a uniform axial field: a uniform density has zero
    drift/diffusion divergence (KAT of the flux form)."""
    pb = workloads.plain(nr=16, nz=24, ion_mass=1.0, seed=0)
    pb.model.reactions = []
    for s in range(2):
        pb.dens[0][s][...] = 0.37
    port = port_tree(pb)
    port.calc_field()
    port.call("port_calc_d_dens_grid")
    for s in range(2):
        assert np.max(np.abs(port.array(0, "d_dens", s))) < 1e-13


def test_r_weighted_mass_conservation():
    """Zero field, no reactions, Neumann boundaries: the divergence telescopes,
    so sum_i r_i n_i is conserved step after step (to rounding)."""
    pb = workloads.plain(nr=24, nz=32, ion_mass=1.0, noise=0.05, seed=3)
    pb.model.reactions = []
    pb.params.E0_z = 0.0
    port = port_tree(pb)
    sp = pb.specs[0]
    r = (np.arange(sp.nr) + 0.5) * pb.params.dr(0)

    def mass():
        return float(np.sum(sp.interior(port.dens(0, 0))[0] * r[None, :]))

    m0 = mass()
    for _ in range(10):
        port.rk2(50.0)
    assert abs(mass() - m0) <= 1e-13 * abs(m0)
