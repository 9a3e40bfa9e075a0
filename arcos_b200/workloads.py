"""Seeded synthetic workloads with the shapes of the five benchmark
configurations (no datasets are involved; every input is generated here).

* single grid (``plain``): the minimal model on an r-z grid, electrons = ions =
  1e-4 + a Gaussian seed of amplitude 0.1, radius 0.1, on the axis at
  z = 0.9 L_z; in 3-D the seed is modulated by 1 + 0.05 cos(theta) +
  0.02 cos(2 theta) and a 1e-6 U[0,1) background is added;
* ``amr``: a refinement tree nested around a seeded streamer-head location;
* ``kinetic``: six charged species, nine tabulated reactions, a batch of
  uneven single-grid instances with their own applied fields.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

from .grids import GridSpec, inherit_ext_bound
from .model import KineticModel, Params, PhotoTerm, Reaction, Species, minimal_model
from .react_table import ReactTable, log_uniform_table


@dataclass
class Problem:
    params: Params
    model: KineticModel
    specs: List[GridSpec]
    dens: List[List[np.ndarray]]                     # [grid][species] rz arrays
    fields: List[Tuple[np.ndarray, np.ndarray, Optional[np.ndarray]]] = field(default_factory=list)
    family_E: List[Tuple[float, float, float]] = field(default_factory=list)

    @property
    def cells(self) -> int:
        return sum(s.nr * s.nz * s.ntheta for s in self.specs)

    @property
    def updated_species(self) -> int:
        """Species a step updates: those with a charge (reaction.c:152) — in
        these models every species."""
        return self.model.no_species


def seed_dens(spec: GridSpec, params: Params, rng: np.random.Generator, amp: float = 0.1,
              sigma: float = 0.1, z_frac: float = 0.9, bg: float = 1e-4,
              noise: float = 0.0, theta_mod: bool = False, center_r: float = 0.0,
              center_z: Optional[float] = None) -> np.ndarray:
    """Density on every cell of ``spec`` (ghosts included) in rz layout."""
    dr, dz = params.dr(spec.level), params.dz(spec.level)
    ir = np.arange(spec.r0 - 2, spec.r1 + 2)
    iz = np.arange(spec.z0 - 2, spec.z1 + 2)
    r = (ir + 0.5) * dr
    z = (iz + 0.5) * dz
    zc = z_frac * params.L_z if center_z is None else center_z
    R, Z = np.meshgrid(r, z)
    g = amp * np.exp(-((R - center_r) ** 2 + (Z - zc) ** 2) / sigma ** 2)
    a = spec.zeros()
    for p in range(spec.planes):
        it = p + spec.theta0
        th = it * params.dtheta
        mod = (1.0 + 0.05 * math.cos(th) + 0.02 * math.cos(2 * th)) if theta_mod else 1.0
        a[p] = bg + g * mod
        if noise > 0:
            a[p] += noise * rng.random(R.shape)
    return a


def uniform_field(spec: GridSpec):
    """The field solve's part of a uniform applied field: zero (the applied
    E0 is added on the device, as cdr_add_ext_field does)."""
    return (spec.zeros(), spec.zeros(), None)


def wavy_field(spec: GridSpec, params: Params, seed: int = 0, e_lo: float = 0.02,
               e_hi: float = 30.0, wavelength: Tuple[float, float] = (14.0, 40.0),
               cancel_applied: bool = True, span: Optional[float] = None):
    """A smooth, non-uniform fixed field: the field solve's part (er, ez,
    None) in rz layout on the staggered points (er at r faces (ir + 1) dr and
    cell-centre z, ez at cell-centre r and z faces (iz + 1) dz; grid.h:40,43).

    Each component is a product of sines with seeded phases and wavelengths
    drawn from ``wavelength`` (in cells of the grid's level), so both
    components change sign inside 32-column and 16-row tiles, and an envelope
    that grows log-uniformly from ``e_lo`` at z = 0 to ``e_hi`` at z = ``span``
    (default L_z), so |E| sweeps a whole reaction table: underflow near
    z = 0, overflow near z = span.  With ``cancel_applied`` the applied E0 is subtracted, so the
    total field (after cdr_add_ext_field adds E0 back) is the wave itself.
    In 3-D each plane is scaled by 1 + 0.3 cos(theta)."""
    rng = np.random.default_rng(seed)
    dr, dz = params.dr(spec.level), params.dz(spec.level)
    ir = np.arange(spec.r0 - 2, spec.r1 + 2, dtype=np.float64)
    iz = np.arange(spec.z0 - 2, spec.z1 + 2, dtype=np.float64)
    lo, hi = wavelength
    k = [2 * math.pi / (float(rng.uniform(lo, hi))) for _ in range(6)]
    ph = [float(rng.uniform(0, 2 * math.pi)) for _ in range(6)]

    top = params.L_z if span is None else span

    def env(zc):
        return e_lo * (e_hi / e_lo) ** np.clip(zc / top, 0.0, 1.0)

    # er: r faces, z centres; ez: r centres, z faces (positions in cells of this level)
    rf, zc = np.meshgrid(ir + 1.0, iz + 0.5)
    rc, zf = np.meshgrid(ir + 0.5, iz + 1.0)
    wr = np.sin(k[0] * rf + ph[0]) * np.cos(k[1] * zc + ph[1]) + 0.4 * np.sin(k[2] * rf + ph[2])
    wz = np.cos(k[3] * rc + ph[3]) * np.sin(k[4] * zf + ph[4]) + 0.4 * np.cos(k[5] * zf + ph[5])
    er2 = env(zc * dz) * wr
    ez2 = env(zf * dz) * wz
    er, ez = spec.zeros(), spec.zeros()
    for p in range(spec.planes):
        th = (p + spec.theta0) * params.dtheta
        mod = 1.0 + 0.3 * math.cos(th) if spec.ntheta > 1 else 1.0
        er[p] = er2 * mod - (params.E0_x if cancel_applied else 0.0)
        ez[p] = ez2 * mod - (params.E0_z if cancel_applied else 0.0)
    return (er, ez, None)


def plain(nr: int = 128, nz: int = 256, ntheta: int = 1, L_r: float = 2.0, L_z: float = 4.0,
          ion_mass: float = 1.0, seed: int = 0, noise: float = 0.0, table_points: int = 256,
          nu: float = 0.5, attempt_dt: float = 50.0, field: str = "uniform") -> Problem:
    """Single uniform grid with the minimal model and a uniform Ez = -1
    (``field="uniform"``), or the non-uniform ``wavy_field`` (``"wavy"``)."""
    params = Params(L_r=L_r, L_z=L_z, gridpoints_r=nr, gridpoints_z=nz, max_ntheta=ntheta,
                    E0_z=-1.0, nu_a=nu, nu_d=nu, nu_rt=nu, diffusion_coeff=0.1,
                    warn_min_timestep=1e-12, max_levels=4)
    model = minimal_model(ion_mass=ion_mass, points=table_points)
    spec = GridSpec(0, 0, nr, nz, ntheta=ntheta, level=0, ext_bound=15, parent=-1)
    rng = np.random.default_rng(seed)
    dens = [[seed_dens(spec, params, rng, noise=noise, theta_mod=ntheta > 1)
             for _ in range(model.no_species)]]
    if field == "wavy":
        fields = [wavy_field(spec, params, seed=seed + 1000)]
    elif field == "uniform":
        fields = [uniform_field(spec)]
    else:
        raise ValueError(f"unknown field {field!r}")
    return Problem(params, model, [spec], dens, fields)


def photo_model(points: int = 256, terms: Sequence[Tuple[float, float]] = ((0.02, -0.8), (0.05, -6.0))
                ) -> KineticModel:
    """The minimal model with photoionization as the reference's kinetic
    reader sets it up (src/rt.c:38-47): electrons, positive ions, the
    counter pair of impact ionization ("dummyplus", the photo source, and
    "dummyminus" to keep the charge balance; react_apply updates charged
    species only, reaction.c:151-153) and the photo ions ("xplus"); impact
    ionization e -> 2e + ion + dummyplus + dummyminus; photo terms (A,
    lambda) in file order."""
    table = log_uniform_table(lambda E: E * math.exp(-1.0 / E), 0.05, 20.0, points)
    return KineticModel(
        species=[Species("electrons", -1.0, 1.0), Species("ions", 1.0, 0.0),
                 Species("dummyplus", 1.0, 0.0), Species("dummyminus", -1.0, 0.0),
                 Species("xplus", 1.0, 0.0)],
        reactions=[Reaction(inputs=[0], outputs=[0, 0, 1, 2, 3], table=table)],
        photo=[PhotoTerm(a, lam) for a, lam in terms],
        photo_source=2, photo_electrons=0, photo_ions=4)


def photo(nr: int = 128, nz: int = 256, ntheta: int = 1, seed: int = 0, noise: float = 0.0,
          field: str = "uniform", terms: Sequence[Tuple[float, float]] = ((0.02, -0.8), (0.05, -6.0))
          ) -> Problem:
    """A single grid with ``photo_model``: a seeded electron/ion cloud, the
    counter and photo species starting at zero, uniform Ez = -1 or the wavy
    field."""
    params = Params(L_r=2.0, L_z=4.0, gridpoints_r=nr, gridpoints_z=nz, max_ntheta=ntheta,
                    E0_z=-1.0, nu_a=0.5, nu_d=0.5, nu_rt=0.5, diffusion_coeff=0.1,
                    warn_min_timestep=1e-12, max_levels=4)
    model = photo_model(terms=terms)
    spec = GridSpec(0, 0, nr, nz, ntheta=ntheta, level=0, ext_bound=15, parent=-1)
    rng = np.random.default_rng(seed)
    dens = [[seed_dens(spec, params, rng, noise=noise, theta_mod=ntheta > 1) for _ in range(2)]
            + [spec.zeros() for _ in range(3)]]
    if field == "wavy":
        fields = [wavy_field(spec, params, seed=seed + 1000)]
    elif field == "uniform":
        fields = [uniform_field(spec)]
    else:
        raise ValueError(f"unknown field {field!r}")
    return Problem(params, model, [spec], dens, fields)


def amr(n_patches: int = 320, levels: int = 4, root_nr: int = 512, root_nz: int = 1024,
        side_lo: int = 16, side_hi: int = 256, seed: int = 0, ion_mass: float = 1.0,
        ntheta: int = 1) -> Problem:
    """A refinement tree of ``n_patches`` patches on ``levels`` levels (ratio
    2) nested around a seeded head point: each level-l patch lies inside one
    level-(l-1) patch (one cell of margin), siblings do not overlap, sides are
    drawn from U{side_lo..side_hi} (clipped to what fits), all even so
    children stay aligned with parent cells."""
    rng = np.random.default_rng(seed)
    params = Params(L_r=2.0, L_z=4.0, gridpoints_r=root_nr, gridpoints_z=root_nz,
                    max_ntheta=ntheta, E0_z=-1.0, nu_a=0.5, nu_d=0.5, nu_rt=0.5,
                    diffusion_coeff=0.1, warn_min_timestep=1e-14, max_levels=levels + 1)
    model = minimal_model(ion_mass=ion_mass)
    specs = [GridSpec(0, 0, root_nr, root_nz, ntheta, 0, 15, -1)]
    head_r = 0.0
    head_z = float(rng.uniform(0.55, 0.85)) * params.L_z
    occupied = {0: []}

    def fits(rect, lst):
        r0, z0, r1, z1 = rect
        for (a0, b0, a1, b1) in lst:
            if r0 < a1 + 2 and a0 < r1 + 2 and z0 < b1 + 2 and b0 < z1 + 2:
                return False
        return True

    target = n_patches - 1
    per_level = []
    rem = target
    weights = [2 ** l for l in range(1, levels)]
    for i, w in enumerate(weights):
        k = rem if i == len(weights) - 1 else int(round(target * w / sum(weights)))
        per_level.append(k)
        rem -= k
    carry = 0
    for l, want in zip(range(1, levels), per_level):
        want += carry
        parents = [i for i, s in enumerate(specs) if s.level == l - 1]
        made = 0
        attempts = 0
        while made < want and attempts < 20000 * max(1, want):
            attempts += 1
            # prefer parents near the head
            pi = parents[int(rng.integers(len(parents)))]
            P = specs[pi]
            pr0, pz0, pr1, pz1 = 2 * P.r0, 2 * P.z0, 2 * P.r1, 2 * P.z1
            wr = int(rng.integers(side_lo, side_hi + 1)) // 2 * 2
            wz = int(rng.integers(side_lo, side_hi + 1)) // 2 * 2
            wr = min(wr, (pr1 - pr0 - 4) // 2 * 2)
            wz = min(wz, (pz1 - pz0 - 4) // 2 * 2)
            if wr < side_lo or wz < side_lo:
                continue
            dr_l = params.dr(l)
            dz_l = params.dz(l)
            cr = int(head_r / dr_l) + int(rng.normal(0, 3 * wr))
            cz = int(head_z / dz_l) + int(rng.normal(0, 3 * wz))
            r0 = min(max(cr - wr // 2, pr0 + 2), pr1 - 2 - wr) // 2 * 2
            z0 = min(max(cz - wz // 2, pz0 + 2), pz1 - 2 - wz) // 2 * 2
            if P.r0 == 0 and rng.random() < 0.3:
                r0 = 0
            r0, z0 = max(r0, pr0 if P.r0 == 0 else pr0 + 2), max(z0, pz0 + 2)
            r1, z1 = r0 + wr, z0 + wz
            if r1 > pr1 - (0 if (P.ext_bound & 2) else 2) or z1 > pz1 - 2:
                continue
            if r0 != 0 and r0 < 2:
                continue
            rect = (r0, z0, r1, z1)
            lst = occupied.setdefault(l, [])
            if not fits(rect, lst):
                continue
            child = GridSpec(r0, z0, r1, z1, ntheta, l, 0, pi)
            child.ext_bound = inherit_ext_bound(P, child)
            specs.append(child)
            lst.append(rect)
            made += 1
        carry = want - made
    dens = []
    for sp in specs:
        per = []
        for s in range(model.no_species):
            per.append(seed_dens(sp, params, rng, noise=1e-6, theta_mod=ntheta > 1,
                                 center_r=head_r, center_z=head_z))
        dens.append(per)
    return Problem(params, model, specs, dens, [uniform_field(s) for s in specs])


def kinetic_model(points: int = 1000, seed: int = 0) -> KineticModel:
    """Six charged species (e, N2+, O2+, O2-, O-, cluster+) and nine reactions
    with seeded smooth monotone rate curves tabulated on ``points``
    log-uniform nodes of [0.01, 50]: impact ionisation of N2 and O2,
    two- and three-body attachment, detachment, two recombinations and ion
    conversion.  Electrons have mass 1, ions mass 100 (mobility 0.01)."""
    rng = np.random.default_rng(seed)
    sp = [Species("e", -1.0, 1.0), Species("N2+", 1.0, 100.0), Species("O2+", 1.0, 100.0),
          Species("O2-", -1.0, 100.0), Species("O-", -1.0, 100.0), Species("X+", 1.0, 100.0)]
    e, n2p, o2p, o2m, om, xp = range(6)

    def curve(kind):
        a = float(rng.uniform(0.5, 2.0))
        b = float(rng.uniform(0.5, 3.0))
        c = float(rng.uniform(0.05, 0.5))
        if kind == "ion":
            return lambda E: a * E * math.exp(-b / E)
        if kind == "att":
            return lambda E: c * a * math.exp(-E / (b * 10.0)) + 1e-3
        return lambda E: c * (1.0 + a * E / (E + b))

    def tab(kind):
        return log_uniform_table(curve(kind), 0.01, 50.0, points)

    reactions = [
        Reaction([e], [e, e, n2p], tab("ion")),       # e + N2 -> 2e + N2+
        Reaction([e], [e, e, o2p], tab("ion")),       # e + O2 -> 2e + O2+
        Reaction([e], [o2m], tab("att")),             # e + O2 + M -> O2- + M
        Reaction([e], [om], tab("att")),              # e + O2 -> O- + O
        Reaction([o2m], [e], tab("det")),             # O2- -> e + O2
        Reaction([e, n2p], [], tab("det")),           # e + N2+ -> N2
        Reaction([o2m, o2p], [], tab("det")),         # O2- + O2+ -> 2 O2
        Reaction([o2p], [xp], tab("det")),            # O2+ + M -> X+
        Reaction([om, xp], [], tab("det")),           # O- + X+ -> neutrals
    ]
    return KineticModel(species=sp, reactions=reactions)


def kinetic_batch(n_inst: int = 32, seed: int = 0, points: int = 1000,
                  sizes_r: Sequence[int] = (64, 128, 256),
                  sizes_z: Sequence[int] = (128, 256, 512), field: str = "uniform") -> Problem:
    """A batch of independent single-grid instances of uneven sizes, each its
    own family with its own applied field Ez ~ U[-2, -0.5].  With
    ``field="wavy"`` each instance also gets a ``wavy_field`` (added to its
    applied field) whose envelope grows from 0.005 at z = 0 to 80 at z = L_z:
    over the default 32 instances |E| reaches both ends of the rate tables
    ([0.01, 50]), while an instance much shorter than L_z stays near its
    applied field.  ``field="wavy_full"`` grows the same envelope over each
    instance's own height, with the instance's applied field subtracted (the
    total field is the wave itself), so every instance, however short,
    sweeps from below the tables' first node to above their last."""
    rng = np.random.default_rng(seed)
    model = kinetic_model(points=points, seed=seed + 1)
    params = Params(L_r=2.0, L_z=4.0, gridpoints_r=128, gridpoints_z=256, E0_z=-1.0,
                    nu_a=0.5, nu_d=0.5, nu_rt=0.5, diffusion_coeff=0.1,
                    warn_min_timestep=1e-14, max_levels=4)
    specs, dens, fields, famE = [], [], [], []
    for i in range(n_inst):
        nr = int(rng.choice(sizes_r))
        nz = int(rng.choice(sizes_z))
        sp = GridSpec(0, 0, nr, nz, 1, 0, 15, -1)
        specs.append(sp)
        # every instance uses the level-0 spacing of the shared params
        per = []
        for s in range(model.no_species):
            amp = 0.1 if s in (0, 1, 2) else 0.01
            per.append(seed_dens(sp, params, rng, amp=amp, noise=1e-6,
                                 center_z=0.9 * nz * params.dz(0)))
        dens.append(per)
        if field in ("wavy", "wavy_full"):
            fields.append(wavy_field(sp, params, seed=seed * 1000 + i, e_lo=0.005, e_hi=80.0,
                                     cancel_applied=False,
                                     span=nz * params.dz(0) if field == "wavy_full" else None))
        elif field == "uniform":
            fields.append(uniform_field(sp))
        else:
            raise ValueError(f"unknown field {field!r}")
        famE.append((0.0, 0.0, float(rng.uniform(-2.0, -0.5))))
        if field == "wavy_full":
            fields[-1][1][...] -= famE[-1][2]     # the total field is the wave itself
    return Problem(params, model, specs, dens, fields, famE)
