"""Discrete adjoint of the fused RK2 CDR step (host side of the C ABI's
arcos_adj_* entry points).

The forward map is the device's fused step (division-free Koren limiter,
fixed field, single-grid 2-D families) with the step sizes frozen to a
recorded sequence, so the map is differentiable away from the limiter's
switch points.  The reverse sweep recomputes each segment of ``ckpt_every``
steps from its checkpoint and applies the transposed step (adjoint_kernel.cuh):

    lam*  = J_F(n*)^T (h/2 lam1)
    lam0  = [n0 > 0] (lam1 + lam* + J_F(max(0, n0))^T (h/2 lam1 + h lam*))

Parameters differentiated: the initial densities, the mobility 1/mass of each
mobile species, diffusion_coeff and every reaction-table value (plus the
under/overflow values).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Dict, List, Optional

import numpy as np

from ._lib import check
from .cdr import CdrTree, _dp


@dataclass
class AdjointGrads:
    dens0: List[List[np.ndarray]]       # [grid][species] dJ/dn(0), rz layout
    mobility: np.ndarray                # [species] dJ/d(1/mass)
    diffusion: float                    # dJ/d diffusion_coeff
    tables: List[np.ndarray]            # [reaction] dJ/d values[0..steps]
    underflow: np.ndarray               # [reaction]
    overflow: np.ndarray                # [reaction]


class Adjoint:
    """Forward with checkpoints and reverse sweep on a committed CdrTree."""

    def __init__(self, tree: CdrTree):
        self.tree = tree
        self.L = tree.L
        self.nsteps = 0
        self.hs: Optional[np.ndarray] = None

    @property
    def n_families(self) -> int:
        return sum(1 for s in self.tree.specs if s.parent < 0)

    def forward(self, nsteps: int, ckpt_every: int = 8, h: float = 1e300,
                h_seq: Optional[np.ndarray] = None) -> np.ndarray:
        """Runs ``nsteps`` steps from the current state; with ``h_seq``
        (families x nsteps) the step sizes are frozen to it, otherwise they
        follow the CFL rule with attempted step ``h``.  Returns the sizes."""
        nf = self.n_families
        hs = np.zeros((nf, nsteps))
        seq = None
        if h_seq is not None:
            seq = np.ascontiguousarray(np.broadcast_to(np.asarray(h_seq, dtype=np.float64), (nf, nsteps)))
        check(self.L.arcos_adj_forward(self.tree.h, nsteps, ckpt_every, h,
                                       _dp(seq) if seq is not None else None, _dp(hs)))
        self.nsteps = nsteps
        self.hs = hs
        return hs

    def set_cotangent(self, gid: int, s: int, lam: np.ndarray):
        a = np.ascontiguousarray(lam, dtype=np.float64)
        assert a.size == int(np.prod(self.tree.specs[gid].shape))
        check(self.L.arcos_adj_set_cotangent(self.tree.h, self.tree.ids[gid], s, _dp(a)))

    def get_cotangent(self, gid: int, s: int) -> np.ndarray:
        a = self.tree.specs[gid].zeros()
        check(self.L.arcos_adj_get_cotangent(self.tree.h, self.tree.ids[gid], s, _dp(a)))
        return a

    def backward(self) -> AdjointGrads:
        m = self.tree.model
        ns = m.no_species
        gm = np.zeros(ns)
        gd = C.c_double(0.0)
        nt = self.L.arcos_adj_table_entries(self.tree.h)
        gt = np.zeros(max(nt, 1))
        check(self.L.arcos_adj_backward(self.tree.h, _dp(gm), C.byref(gd), _dp(gt)))
        nre = len(m.reactions)
        tables, under, over = [], np.zeros(nre), np.zeros(nre)
        n_nodes = nt - 2 * nre
        for r, re in enumerate(m.reactions):
            off = self.L.arcos_adj_table_offset(self.tree.h, r)
            tables.append(gt[off:off + re.table.steps + 1].copy())
            under[r] = gt[n_nodes + 2 * r]
            over[r] = gt[n_nodes + 2 * r + 1]
        dens0 = [[self.get_cotangent(g, s) for s in range(ns)] for g in range(len(self.tree.specs))]
        return AdjointGrads(dens0, gm, gd.value, tables, under, over)


def smooth_direction(rng: np.random.Generator, nz: int, nr: int, modes: int = 4) -> np.ndarray:
    """A seeded smooth random field on nz x nr cells (a few low Fourier
    modes), the finite-difference check's direction for densities: it moves
    the limiter's upwind differences far less than white noise would, so a
    1e-6 step stays away from the limiter's switch points."""
    z = (np.arange(nz) + 0.5) / nz
    r = (np.arange(nr) + 0.5) / nr
    f = np.zeros((nz, nr))
    for _ in range(modes):
        kz, kr = rng.integers(1, 4, size=2)
        f += rng.standard_normal() * np.cos(np.pi * kz * z + rng.uniform(0, 2 * np.pi))[:, None] \
            * np.cos(np.pi * kr * r + rng.uniform(0, 2 * np.pi))[None, :]
    return f


def fd_objective_difference(ne_p: np.ndarray, ne_m: np.ndarray, target: np.ndarray,
                            vol: np.ndarray, eps: float) -> float:
    """Central difference (J(+) - J(-)) / (2 eps) of J = 1/2 sum vol (n - t)^2,
    written as 1/2 sum vol (a - b)(a + b - 2t) so the objectives never cancel."""
    return 0.5 * float(np.sum(vol * (ne_p - ne_m) * (ne_p + ne_m - 2.0 * target))) / (2 * eps)


def cell_volume(spec, dr: float, dz: float) -> np.ndarray:
    """2 pi r_i dr dz of every cell of a 2-D grid (rz layout, ghosts 0)."""
    v = np.zeros(spec.shape)
    r = (np.arange(spec.r0, spec.r1) + 0.5) * dr
    v[0, 2:-2, 2:-2] = (2.0 * np.pi * r * dr * dz)[None, :]
    return v
