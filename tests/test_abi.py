"""The C ABI library: loads without a GPU, exports every function that
include/arcos_cdr.h declares, rejects bad arguments before touching CUDA,
and its host-side table lookup is the reference's lookup exactly."""
import ctypes as C
import math
import os
import re

import numpy as np
import pytest

from arcos_b200 import _lib
from arcos_b200.react_table import log_uniform_table, minimal_alpha

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "arcos_cdr.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:int|void|const\s+char\s*\*)\s*\**\s*(arcos_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) >= 40
    lib = C.CDLL(_lib.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_create_rejects_bad_species_count_without_cuda():
    L = _lib.lib()
    p = _lib.ArcosParams()
    p.no_species = 0
    p.max_ntheta = 1
    h = C.c_void_p()
    rc = L.arcos_create(C.byref(p), C.byref(h))
    assert rc == 1
    assert b"no_species" in L.arcos_last_error()
    p.no_species = 2
    p.max_ntheta = 0
    assert L.arcos_create(C.byref(p), C.byref(h)) == 1


def reference_rate(t, e):
    """react_apply's lookup (reaction.c:127-142), evaluated with the host libm."""
    log_e = math.log10(e) if e > 0 else -math.inf
    if log_e < t.e_min:
        return t.underflow
    if log_e > t.e_min + t.e_step * t.steps:
        return t.overflow
    pos = math.floor((log_e - t.e_min) / t.e_step)
    v = t.padded_values()
    e1 = math.pow(10, t.e_min + t.e_step * pos)
    e2 = e1 * math.pow(10, t.e_step)
    return v[pos] + ((v[pos + 1] - v[pos]) / (e2 - e1)) * (e - e1)


def table_rates(t, e):
    L = _lib.lib()
    L.arcos_table_rates.argtypes = [C.c_double, C.c_double, C.c_int, C.c_double, C.c_double,
                                    _lib.DP, _lib.DP, C.c_int, _lib.DP]
    v = np.ascontiguousarray(t.values, dtype=np.float64)
    e = np.ascontiguousarray(e, dtype=np.float64)
    out = np.zeros_like(e)
    _lib.check(L.arcos_table_rates(t.e_min, t.e_step, t.steps, t.underflow, t.overflow,
                                   v.ctypes.data_as(_lib.DP), e.ctypes.data_as(_lib.DP), e.size,
                                   out.ctypes.data_as(_lib.DP)))
    return out


@pytest.mark.parametrize("points,lo,hi", [(256, 0.05, 20.0), (1000, 0.01, 50.0), (4, 0.01, 10.0)])
def test_table_lookup_is_exact(points, lo, hi):
    """The device replaces log10/floor by exact per-node thresholds; on random
    fields and on every node position (where floor decides the segment) the
    rate must be bit-identical to the reference formula."""
    t = log_uniform_table(minimal_alpha, lo, hi, points)
    rng = np.random.default_rng(points)
    e = np.concatenate([
        10.0 ** rng.uniform(math.log10(lo) - 1, math.log10(hi) + 1, 4000),
        [10.0 ** (t.e_min + t.e_step * k) for k in range(points)],
        [np.nextafter(10.0 ** (t.e_min + t.e_step * k), 0) for k in range(points)],
        [np.nextafter(10.0 ** (t.e_min + t.e_step * k), np.inf) for k in range(points)],
        [0.0, lo, hi, 1e300, 1.0],
    ])
    got = table_rates(t, e)
    want = np.array([reference_rate(t, x) for x in e])
    assert np.array_equal(got, want)
