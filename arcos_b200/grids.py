"""Grid (patch) descriptors and the rz_array host layout.

A grid covers cells ``[r0, r1) x [z0, z1)`` at refinement ``level`` (cell
indices are absolute at that level), plus two ghost cells on each side, with
``ntheta`` azimuthal planes (include/cdr.h:22-42, include/grid.h:10).  Host
arrays use the reference layout (src/rz_array.c:23-96): numpy shape
``(planes, nz + 4, nr + 4)`` in C order, so r is the fastest index;
``planes`` is 1 for ntheta == 1 and ntheta + 4 otherwise (theta from -2).

``ext_bound`` is the mask of sides on the domain boundary (grid.h:22-31) and
``parent`` the index of the parent grid in the list (-1 for the root).  Sibling
order follows tree.h's add_child, which prepends: the reference visits the
children of a grid in the reverse of their creation order.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Sequence

import numpy as np

from .model import BND_MASK_BOTTOM, BND_MASK_LEFT, BND_MASK_RIGHT, BND_MASK_TOP


@dataclass
class GridSpec:
    r0: int
    z0: int
    r1: int
    z1: int
    ntheta: int = 1
    level: int = 0
    ext_bound: int = 15
    parent: int = -1

    @property
    def nr(self) -> int:
        return self.r1 - self.r0

    @property
    def nz(self) -> int:
        return self.z1 - self.z0

    @property
    def planes(self) -> int:
        return 1 if self.ntheta == 1 else self.ntheta + 4

    @property
    def theta0(self) -> int:
        return 0 if self.ntheta == 1 else -2

    @property
    def shape(self):
        return (self.planes, self.nz + 4, self.nr + 4)

    def zeros(self) -> np.ndarray:
        return np.zeros(self.shape, dtype=np.float64)

    def interior(self, a: np.ndarray) -> np.ndarray:
        """View of the real cells (all real planes for 3-D arrays)."""
        t0 = 0 - self.theta0
        return a[t0:t0 + self.ntheta, 2:self.nz + 2, 2:self.nr + 2]


def inherit_ext_bound(parent: GridSpec, child: GridSpec) -> int:
    """grid_inherit_ext_bound (src/grid.c:205-235)."""
    eb = 0
    if parent.ext_bound == 0:
        return 0
    if parent.ext_bound & BND_MASK_LEFT and (parent.r0 << 1) == child.r0:
        eb |= BND_MASK_LEFT
    if parent.ext_bound & BND_MASK_RIGHT and (parent.r1 << 1) == child.r1:
        eb |= BND_MASK_RIGHT
    if parent.ext_bound & BND_MASK_BOTTOM and (parent.z0 << 1) == child.z0:
        eb |= BND_MASK_BOTTOM
    if parent.ext_bound & BND_MASK_TOP and (parent.z1 << 1) == child.z1:
        eb |= BND_MASK_TOP
    return eb


def children_in_visit_order(specs: Sequence[GridSpec], gid: int) -> List[int]:
    """Child indices of grid ``gid`` in the order iter_childs visits them."""
    kids = [i for i, s in enumerate(specs) if s.parent == gid]
    return kids[::-1]
