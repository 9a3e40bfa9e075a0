"""Reaction-rate tables k(|E|) in the arcos text format.

Mirrors ``react_table`` (include/react_table.h:9-20) and ``react_table_read``
(src/react_table.c:73-111): everything up to a line starting with ``START`` is
ignored, then come ``e_min`` (log10 of the lowest field), ``e_step`` (log10
spacing), ``points``, ``underflow``, ``overflow`` and ``points`` values.  As in
the reference, ``steps = points - 1`` and there is no ``is_log`` line (the
comment at react_table.c:12-20 mentions one, the parser does not read it).

The reference stores at most MAX_TABLE_SIZE = 500 values (react_table.h:5) and
does not check it; this module has no such limit.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np


@dataclass
class ReactTable:
    e_min: float
    e_step: float
    steps: int
    underflow: float
    overflow: float
    values: np.ndarray = field(repr=False)

    @property
    def points(self) -> int:
        return self.steps + 1

    def padded_values(self) -> np.ndarray:
        """``steps + 2`` values: the lookup at ``pos == steps`` (a field exactly
        at the top node) reads ``values[steps + 1]``, which the reference leaves
        uninitialised (reaction.c:136-141); it repeats ``values[steps]`` here."""
        v = np.asarray(self.values, dtype=np.float64)
        return np.concatenate([v, v[-1:]])


def react_table_read(path: str | os.PathLike) -> ReactTable:
    """Parse a table file with the semantics of react_table.c:73-111
    (``atof``/``atoi`` on successive lines after ``START``).  Where the
    reference exits (missing file: FileNotFoundError here) or reads garbage
    (no START line: it loops forever; a truncated file: it repeats the last
    line; fewer than 2 points or e_step <= 0: a table the lookup cannot use)
    this reader raises."""
    with open(path, "r") as fp:
        lines = fp.read().splitlines()
    i = 0
    while i < len(lines) and not lines[i].startswith("START"):
        i += 1
    if i >= len(lines):
        raise ValueError(f"{path}: no START line")

    def atof(s: str) -> float:
        s = s.strip()
        num = ""
        for ch in s:
            if ch in "0123456789+-.eE":
                num += ch
            else:
                break
        try:
            return float(num)
        except ValueError:
            return 0.0

    vals = lines[i + 1:]
    if len(vals) < 5:
        raise ValueError(f"{path}: the header after START needs 5 lines, found {len(vals)}")
    e_min = atof(vals[0])
    e_step = atof(vals[1])
    steps = int(atof(vals[2])) - 1
    underflow = atof(vals[3])
    overflow = atof(vals[4])
    if steps < 1:
        raise ValueError(f"{path}: a table needs at least 2 points, found {steps + 1}")
    if not (e_step > 0):
        raise ValueError(f"{path}: e_step must be positive, found {e_step}")
    values = np.array([atof(v) for v in vals[5:5 + steps + 1]], dtype=np.float64)
    if values.size != steps + 1:
        raise ValueError(f"{path}: expected {steps + 1} values, found {values.size}")
    return ReactTable(e_min, e_step, steps, underflow, overflow, values)


def write_react_table(path: str | os.PathLike, table: ReactTable, comment: str = "") -> None:
    """Write ``table`` in the format react_table_read parses, with every number
    printed with 17 significant digits so it reads back bit for bit."""
    with open(path, "w") as fp:
        if comment:
            fp.write(comment.rstrip("\n")[:99] + "\n")
        fp.write("START\n")
        fp.write(f"{table.e_min:.17g}\n{table.e_step:.17g}\n{table.points}\n")
        fp.write(f"{table.underflow:.17g}\n{table.overflow:.17g}\n")
        for v in np.asarray(table.values, dtype=np.float64):
            fp.write(f"{v:.17g}\n")


def log_uniform_table(fn, e_lo: float, e_hi: float, points: int) -> ReactTable:
    """A table of ``fn(E)`` on ``points`` log-uniform nodes of [e_lo, e_hi];
    under/overflow are the end values.  The node positions are the ones the
    lookup reconstructs, ``10**(e_min + e_step*pos)``."""
    e_min = math.log10(e_lo)
    e_step = (math.log10(e_hi) - e_min) / (points - 1)
    nodes = [10.0 ** (e_min + e_step * k) for k in range(points)]
    values = np.array([fn(e) for e in nodes], dtype=np.float64)
    return ReactTable(e_min, e_step, points - 1, float(values[0]), float(values[-1]), values)


def minimal_alpha(e: float) -> float:
    """Impact-ionisation coefficient of the arcos minimal model,
    alpha(|E|) = |E| exp(-1/|E|)."""
    return e * math.exp(-1.0 / e) if e > 0 else 0.0
