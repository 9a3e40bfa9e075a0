"""Kinetic model and run parameters: the host-side state the reference keeps in
globals (include/parameters.h:24-61, include/species.h:12-20,
include/reaction.h:13-46, src/cstream.c:276-306) gathered into plain objects.

``Species.mass`` follows the reference convention: mobility is ``1/mass`` and
``mass <= 0`` means immobile (species.h:14).  Reactions are kept in list order,
which is the order react_apply_all applies them (reaction.c:203-210; the
kinetic reader adds them so that the list is in file order, rt.c:46-47).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Sequence

from .react_table import ReactTable, log_uniform_table, minimal_alpha

# Boundary numbering and masks of include/grid.h:14-31.
BND_LEFT, BND_RIGHT, BND_BOTTOM, BND_TOP = 0, 1, 2, 3
BND_MASK_LEFT, BND_MASK_RIGHT, BND_MASK_BOTTOM, BND_MASK_TOP = 1, 2, 4, 8
BND_MASK_ALL = 15
BND_CND_HNEUMANN, BND_CND_HDIRICHLET = 1, -1   # include/rz_array.h:71-72


@dataclass
class Species:
    name: str
    charge: float
    mass: float


@dataclass
class Reaction:
    inputs: Sequence[int]
    outputs: Sequence[int]
    table: ReactTable


@dataclass
class Params:
    """The globals the density update reads (defaults from
    init_parameters, src/cstream.c:54-269, where they matter here)."""
    L_r: float = 2.0
    L_z: float = 4.0
    gridpoints_r: int = 128
    gridpoints_z: int = 256
    max_ntheta: int = 1
    max_levels: int = 8
    extra_pois_levels: int = 2
    diffusion_coeff: float = 0.1
    nu_a: float = 0.2
    nu_d: float = 0.2
    nu_rt: float = 0.2
    E0_x: float = 0.0
    E0_y: float = 0.0
    E0_z: float = -0.06
    cdr_bnd_bottom: int = BND_CND_HNEUMANN
    cdr_bnd_top: int = BND_CND_HNEUMANN
    cdr_bnd_right: int = BND_CND_HNEUMANN
    warn_min_timestep: float = 1e-6
    z_cutoff: float = 1e7        # src/cdr.c:37
    per_plane: bool = True       # drift/diffusion on every theta plane (3-D)

    def dr(self, level: int) -> float:
        return self.grid_sizes()[0][level]

    def dz(self, level: int) -> float:
        return self.grid_sizes()[1][level]

    def grid_sizes(self):
        """dr[], dz[] per level with the arithmetic of init_gridsizes_a
        (src/cstream.c:276-306): start ``extra_pois_levels`` levels coarser and
        halve; level 0 is index ``extra_pois_levels``."""
        n = self.max_levels + self.extra_pois_levels + 1
        root_dr = self.L_r / self.gridpoints_r
        root_dz = self.L_z / self.gridpoints_z
        drs = [root_dr * (1 << self.extra_pois_levels)]
        dzs = [root_dz * (1 << self.extra_pois_levels)]
        for _ in range(1, n):
            drs.append(drs[-1] / 2.0)
            dzs.append(dzs[-1] / 2.0)
        e = self.extra_pois_levels
        return drs[e:], dzs[e:]

    @property
    def dtheta(self) -> float:
        return 6.283185307179586477 / self.max_ntheta   # twopi, cstream.c:38


@dataclass
class PhotoTerm:
    """One term of the photoionization file (photo_load_file,
    src/photo.c:373-400): the source weight A and the Helmholtz shift lambda
    (passed as ES to the solver, src/photo.c:296-305)."""
    A: float
    lam: float


@dataclass
class KineticModel:
    species: List[Species] = field(default_factory=list)
    reactions: List[Reaction] = field(default_factory=list)
    # Photoionization (has_photoionization, src/rt.c:38-47): terms in file
    # order (photo_calc visits them last-first, photo_register prepends,
    # src/photo.c:174-185); the source species ("dummyplus", whose d_dens is
    # the impact ionization rate), and the two species that receive A * photo
    # ("electrons" and "xplus", src/photo.c:268-291).  The photo entry ends
    # the reactions list.
    photo: List[PhotoTerm] = field(default_factory=list)
    photo_source: int = -1
    photo_electrons: int = 0
    photo_ions: int = -1

    @property
    def no_species(self) -> int:
        return len(self.species)


def minimal_model(ion_mass: float = 0.0, points: int = 256, e_lo: float = 0.05,
                  e_hi: float = 20.0) -> KineticModel:
    """Electrons (charge -1, mass 1) and positive ions (charge +1, mass
    ``ion_mass``; 0 = immobile) with impact ionisation e -> 2e + ion, whose
    rate alpha(|E|) = |E| exp(-1/|E|) is tabulated on ``points`` log-uniform
    nodes of [e_lo, e_hi]."""
    table = log_uniform_table(minimal_alpha, e_lo, e_hi, points)
    return KineticModel(
        species=[Species("electrons", -1.0, 1.0), Species("ions", 1.0, ion_mass)],
        reactions=[Reaction(inputs=[0], outputs=[0, 0, 1], table=table)],
    )
