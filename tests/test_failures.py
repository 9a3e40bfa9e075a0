"""Failure detection, injected on the host (no GPU fault is ever caused):

* a density that is NaN everywhere makes the CFL maxima invalid - the
  assertion of cdr_courant (src/cdr.c:1023) - and the step reports
  ARCOS_ERR_NAN;
* a warn_min_timestep above the CFL step: the reference warns five times and
  stops at the sixth small step (src/cdr.c:1269,1296-1302); the device steps
  report ARCOS_ERR_SMALL_DT on the sixth;
* a corrupt or truncated reaction-table file is refused by the reader
  (src/react_table.c:73-111 exits on a missing file and otherwise reads
  whatever is there, or loops forever without a START line);
* degenerate grids and impossible trees are refused before any launch.

After each error the context stays usable: fresh inputs step normally.
The CPU tests need no device; the rest run on the GPU with valid launches
only (the errors come from the data, not from the kernels).
"""
import ctypes as C
import os

import numpy as np
import pytest

from arcos_b200 import workloads
from arcos_b200._lib import ArcosError, ArcosParams, lib
from arcos_b200.cdr import CdrTree
from arcos_b200.react_table import react_table_read, write_react_table, log_uniform_table
from arcos_b200.react_table import minimal_alpha

ERR_ARG, ERR_NAN, ERR_SMALL_DT = 1, 3, 4


# ------------------------------------------------------------------ CPU ----
def test_missing_table_file_is_refused(tmp_path):
    with pytest.raises(FileNotFoundError):
        react_table_read(tmp_path / "absent.reaction")


def test_table_without_start_is_refused(tmp_path):
    p = tmp_path / "nostart.reaction"
    p.write_text("a comment\n-1.3\n0.01\n3\n0\n1\n0.1\n0.2\n0.3\n")
    with pytest.raises(ValueError, match="START"):
        react_table_read(p)


def test_truncated_table_is_refused(tmp_path):
    t = log_uniform_table(minimal_alpha, 0.05, 20.0, 16)
    p = tmp_path / "t.reaction"
    write_react_table(p, t)
    lines = p.read_text().splitlines()
    p.write_text("\n".join(lines[:-3]) + "\n")           # three values missing
    with pytest.raises(ValueError, match="expected 16 values"):
        react_table_read(p)


def test_table_with_too_few_points_is_refused(tmp_path):
    p = tmp_path / "one.reaction"
    p.write_text("START\n-1.3\n0.01\n1\n0\n1\n0.5\n")
    with pytest.raises(ValueError, match="points"):
        react_table_read(p)


def test_create_rejects_bad_species_count_without_a_device():
    """Argument checks of arcos_create come before any CUDA call."""
    L = lib()
    p = ArcosParams()
    p.no_species = 7
    p.max_ntheta = 1
    h = C.c_void_p()
    assert L.arcos_create(C.byref(p), C.byref(h)) == ERR_ARG
    assert b"no_species" in L.arcos_last_error()
    p.no_species = 2
    p.max_ntheta = 0
    assert L.arcos_create(C.byref(p), C.byref(h)) == ERR_ARG


def test_table_rates_rejects_bad_tables_without_a_device():
    L = lib()
    v = np.ones(4)
    e = np.ones(2)
    out = np.zeros(2)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))   # noqa: E731
    assert L.arcos_table_rates(C.c_double(-1.0), C.c_double(0.0), 3, C.c_double(0), C.c_double(1),
                               dp(v), dp(e), 2, dp(out)) == ERR_ARG
    assert L.arcos_table_rates(C.c_double(-1.0), C.c_double(0.1), 0, C.c_double(0), C.c_double(1),
                               dp(v), dp(e), 2, dp(out)) == ERR_ARG


# ------------------------------------------------------------------ GPU ----
def _tree(pb, exact=False):
    t = CdrTree(pb.params, pb.model, pb.specs, exact=exact)
    for g, per in enumerate(pb.dens):
        for s, a in enumerate(per):
            t.upload(g, "dens", a, s)
    t.set_fixed_field(pb.fields)
    return t


@pytest.mark.gpu
@pytest.mark.parametrize("exact", [False, True])
def test_nan_density_reports_invalid_cfl_maxima(cuda_device, exact):
    pb = workloads.plain(nr=24, nz=40, ion_mass=1.0, noise=1e-3, seed=1)
    t = _tree(pb, exact=exact)
    nan = np.full(pb.specs[0].shape, np.nan)
    for s in range(2):
        t.upload(0, "dens", nan, s)
    with pytest.raises(ArcosError) as ei:
        t.run(1, 50.0)
    assert ei.value.code == ERR_NAN
    # the context is still usable: valid densities step normally
    t2 = _tree(pb, exact=exact)
    assert t2.run(2, 50.0)[0][0] > 0
    t2.close()
    t.close()


@pytest.mark.gpu
def test_nan_density_tree_step(cuda_device):
    """The same through the grid-level cdr_rk2 entry point."""
    pb = workloads.plain(nr=24, nz=40, ion_mass=1.0, noise=1e-3, seed=2)
    t = _tree(pb, exact=True)
    nan = np.full(pb.specs[0].shape, np.nan)
    for s in range(2):
        t.upload(0, "dens", nan, s)
    with pytest.raises(ArcosError) as ei:
        t.cdr_rk2(50.0)
    assert ei.value.code == ERR_NAN
    t.close()


@pytest.mark.gpu
@pytest.mark.parametrize("exact", [False, True])
def test_small_timestep_stops_at_the_sixth_step(cuda_device, exact):
    pb = workloads.plain(nr=24, nz=40, ion_mass=1.0, noise=1e-3, seed=3)
    pb.params.warn_min_timestep = 1.0          # far above the CFL step (~2e-2)
    t = _tree(pb, exact=exact)
    dts = t.run(5, 50.0)[0]                      # five warnings are tolerated
    assert np.all(dts < 1.0)
    with pytest.raises(ArcosError) as ei:
        t.run(1, 50.0)
    assert ei.value.code == ERR_SMALL_DT
    t.close()


@pytest.mark.gpu
def test_small_timestep_per_call_and_tree_step(cuda_device):
    """Step by step (the step size of the next step is computed ahead and
    again at the next call: it counts once), and through cdr_rk2."""
    pb = workloads.plain(nr=24, nz=40, ion_mass=1.0, noise=1e-3, seed=3)
    pb.params.warn_min_timestep = 1.0
    t = _tree(pb, exact=False)
    for _ in range(5):
        t.run(1, 50.0)
    with pytest.raises(ArcosError) as ei:
        t.run(1, 50.0)
    assert ei.value.code == ERR_SMALL_DT
    t.close()
    t = _tree(pb, exact=True)
    for _ in range(5):
        t.cdr_rk2(50.0)
    with pytest.raises(ArcosError) as ei:
        t.cdr_rk2(50.0)
    assert ei.value.code == ERR_SMALL_DT
    t.close()


@pytest.mark.gpu
def test_degenerate_grids_are_refused_before_any_launch(cuda_device):
    pb = workloads.plain(nr=16, nz=16, ion_mass=1.0, seed=4)
    L = lib()
    from arcos_b200.cdr import make_params
    p = make_params(pb.params, pb.model)
    h = C.c_void_p()
    assert L.arcos_create(C.byref(p), C.byref(h)) == 0
    gid = C.c_int(-1)
    try:
        # zero-size and one-cell patches
        assert L.arcos_grid_new(h, 0, 0, 0, 16, 1, 0, 15, -1, C.byref(gid)) == ERR_ARG
        assert L.arcos_grid_new(h, 0, 0, 16, 1, 1, 0, 15, -1, C.byref(gid)) == ERR_ARG
        # an axis boundary away from the axis
        assert L.arcos_grid_new(h, 4, 0, 16, 16, 1, 0, 15, -1, C.byref(gid)) == ERR_ARG
        # a parent that does not exist, a child two levels down, a child outside its parent
        assert L.arcos_grid_new(h, 0, 0, 8, 8, 1, 1, 0, 3, C.byref(gid)) == ERR_ARG
        assert L.arcos_grid_new(h, 0, 0, 16, 16, 1, 0, 15, -1, C.byref(gid)) == 0
        root = gid.value
        assert L.arcos_grid_new(h, 4, 4, 12, 12, 1, 2, 0, root, C.byref(gid)) == ERR_ARG
        assert L.arcos_grid_new(h, 4, 4, 60, 12, 1, 1, 0, root, C.byref(gid)) == ERR_ARG
        # odd child corners (not aligned with parent cells)
        assert L.arcos_grid_new(h, 4, 5, 12, 12, 1, 1, 0, root, C.byref(gid)) == ERR_ARG
        # nothing to step before commit
        assert L.arcos_run(h, 1, C.c_double(1.0), None) != 0
        assert L.arcos_commit(h) == 0
        # grids cannot be added after commit
        assert L.arcos_grid_new(h, 4, 4, 12, 12, 1, 1, 0, root, C.byref(gid)) != 0
    finally:
        L.arcos_destroy(h)
