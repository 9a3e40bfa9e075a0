"""Shared helpers for the parity tests: run a workload through the CPU oracle
(the restatement in oracle/) and compare arrays."""
from __future__ import annotations

import copy

import numpy as np

from arcos_b200.workloads import Problem
from oracle import bind


def port_tree(pb: Problem, field_mode=bind.FIELD_FIXED, zero_all=True, per_plane=None,
              E=None):
    params = copy.deepcopy(pb.params)
    if per_plane is not None:
        params.per_plane = per_plane
    if E is not None:
        params.E0_x, params.E0_y, params.E0_z = E
    t = bind.PortTree(params, pb.model, pb.specs, field_mode=field_mode, zero_all=zero_all)
    for g, per in enumerate(pb.dens):
        for s, a in enumerate(per):
            t.dens(g, s)[...] = a
    if field_mode == bind.FIELD_FIXED:
        for g, (er, ez, et) in enumerate(pb.fields):
            sp = pb.specs[g]
            t.set_fixed_field(g, er, ez, et if et is not None else sp.zeros())
    return t


def single_family(pb: Problem, i: int) -> Problem:
    """Instance ``i`` of a batch as a problem of its own (one family)."""
    sub = copy.copy(pb)
    sub.specs = [pb.specs[i]]
    sub.dens = [pb.dens[i]]
    sub.fields = [pb.fields[i]]
    sub.family_E = [pb.family_E[i]] if pb.family_E else []
    return sub


def max_ulp(a: np.ndarray, b: np.ndarray) -> int:
    """Largest distance in units in the last place between equal-shape arrays
    (0 means bit-identical up to the sign of zero)."""
    a = np.ascontiguousarray(a, dtype=np.float64).ravel()
    b = np.ascontiguousarray(b, dtype=np.float64).ravel()
    ia = a.view(np.int64).copy()
    ib = b.view(np.int64).copy()
    ia = np.where(ia < 0, np.int64(-0x8000000000000000) - ia, ia)
    ib = np.where(ib < 0, np.int64(-0x8000000000000000) - ib, ib)
    d = np.abs(ia - ib)
    d[(a == b)] = 0
    return int(d.max()) if d.size else 0


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.maximum(np.abs(b), 1e-300)
    return float(np.max(np.abs(a - b) / den)) if a.size else 0.0
