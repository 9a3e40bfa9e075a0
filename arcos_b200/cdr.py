"""Host-side mirror of the reference CDR interface over the device library.

``CdrTree`` holds one grid family (or a batch of independent families) on the
device and exposes the entry points of src/cdr.c and src/reaction.c by their
reference names, each acting on a whole storage set the way the reference's
recursive ``*_r`` variants act on a tree:

=============================  ==============================================
reference (src/cdr.c ...)      CdrTree
=============================  ==============================================
cdr_nonegative_r   :703-721    cdr_nonegative_r(set)
cdr_set_ext_bnd_r  :726-768    cdr_set_ext_bnd_r(set)
cdr_set_periodic_r :288-310    cdr_set_periodic_r(set)
cdr_restrict_r     :2050-2097  cdr_restrict_r(set)
cdr_set_bnd_r      :1888-1948  cdr_set_bnd_r(set)
cdr_match_r        :1763-1882  cdr_match_r(set)
prepare_grid       :1334-1351  prepare_grid(set)
cdr_calc_field_r   :532-580    set_field(...) / field_post(set) / field callback /
                               set_field_poisson (the solve on the device)
cdr_calc_charge_r  :361-389    cdr_calc_charge_r(set)
react_apply_all    reaction.c:192-211   react_apply_all(set)
cdr_advect_diffu_r :900-955    cdr_advect_diffu_r(set)
cdr_calc_d_dens    :830-835    cdr_calc_d_dens(set)
cdr_courant        :971-1061   cdr_courant(set)
cdr_update         :1075-1100  cdr_update(h)         (grid -> inter)
cdr_rk2_update_r   :1107-1162  cdr_rk2_update(h)     (grid, inter -> grid)
cdr_rk2            :1262-1327  cdr_rk2(h)
=============================  ==============================================

Storage set 0 is the reference's ``grid`` tree and set 1 its ``inter`` tree.
Arrays cross the boundary in the rz_array layout (see grids.py).
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, List, Optional, Sequence

import numpy as np

from ._lib import DP, FIELD_FN, ArcosParams, RefineParams, check, lib
from .grids import GridSpec
from .model import KineticModel, Params

DENS, D_DENS, ER, EZ, ETHETA, EABS, CHARGE = range(7)
KINDS = {"dens": DENS, "d_dens": D_DENS, "er": ER, "ez": EZ, "etheta": ETHETA,
         "eabs": EABS, "charge": CHARGE}
SET_GRID, SET_INTER = 0, 1


def _dp(a: np.ndarray):
    return a.ctypes.data_as(DP)


def make_params(params: Params, model: KineticModel) -> ArcosParams:
    p = ArcosParams()
    p.no_species = model.no_species
    for s, sp in enumerate(model.species):
        p.charge[s] = sp.charge
        p.mass[s] = sp.mass
    p.diffusion_coeff = params.diffusion_coeff
    p.nu_a, p.nu_d, p.nu_rt = params.nu_a, params.nu_d, params.nu_rt
    p.warn_min_timestep = params.warn_min_timestep
    p.cdr_bnd_bottom, p.cdr_bnd_top, p.cdr_bnd_right = (params.cdr_bnd_bottom, params.cdr_bnd_top,
                                                        params.cdr_bnd_right)
    p.E_x, p.E_y, p.E_z = params.E0_x, params.E0_y, params.E0_z
    p.z_cutoff = params.z_cutoff
    p.L_r, p.L_z = params.L_r, params.L_z
    p.gridpoints_r, p.gridpoints_z = params.gridpoints_r, params.gridpoints_z
    p.max_ntheta = params.max_ntheta
    p.max_levels = params.max_levels
    p.extra_pois_levels = params.extra_pois_levels
    p.per_plane = 1 if params.per_plane else 0
    return p


class CdrTree:
    """One or more grid families resident on the current CUDA device."""

    def __init__(self, params: Params, model: KineticModel, specs: Sequence[GridSpec],
                 per_patch: bool = False, tile: int = 2, stream: Optional[int] = None,
                 exact: bool = False):
        self.L = lib()
        self.params, self.model, self.specs = params, model, list(specs)
        self._p = make_params(params, model)
        h = C.c_void_p()
        check(self.L.arcos_create(C.byref(self._p), C.byref(h)))
        self.h = h
        if stream is not None:
            check(self.L.arcos_set_stream(self.h, C.c_void_p(stream)))
        for re in model.reactions:
            ins = (C.c_int * max(1, len(re.inputs)))(*re.inputs)
            outs = (C.c_int * max(1, len(re.outputs)))(*re.outputs)
            v = np.ascontiguousarray(re.table.values, dtype=np.float64)
            t = re.table
            check(self.L.arcos_add_reaction(self.h, len(re.inputs), ins, len(re.outputs), outs,
                                            t.e_min, t.e_step, t.steps, t.underflow, t.overflow,
                                            _dp(v)))
        self.ids: List[int] = []
        for sp in self.specs:
            gid = C.c_int(0)
            parent = self.ids[sp.parent] if sp.parent >= 0 else -1
            check(self.L.arcos_grid_new(self.h, sp.r0, sp.z0, sp.r1, sp.z1, sp.ntheta, sp.level,
                                        sp.ext_bound, parent, C.byref(gid)))
            self.ids.append(gid.value)
        check(self.L.arcos_set_tile(self.h, tile))
        check(self.L.arcos_set_exact(self.h, 1 if exact else 0))
        check(self.L.arcos_set_per_patch(self.h, 1 if per_patch else 0))
        check(self.L.arcos_commit(self.h))
        self._field_cb = None
        if model.photo:                         # has_photoionization (rt.c:38-47)
            self.set_photo()

    def close(self):
        if getattr(self, "h", None):
            self.L.arcos_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- data movement (rz layout) ----
    def upload(self, gid: int, what: str, arr: np.ndarray, s: int = 0, set: int = SET_GRID):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        assert a.size == int(np.prod(self.specs[gid].shape)), "array does not match the grid shape"
        check(self.L.arcos_upload(self.h, self.ids[gid], set, KINDS[what], s, _dp(a)))

    def download(self, gid: int, what: str, s: int = 0, set: int = SET_GRID) -> np.ndarray:
        a = self.specs[gid].zeros()
        check(self.L.arcos_download(self.h, self.ids[gid], set, KINDS[what], s, _dp(a)))
        return a

    def dump(self, path, gid: int = 0, what: str = "dens", s: int = 0, set: int = SET_GRID):
        """FP64 dump of one array's interior (rz_dump_3d's order, lossless)."""
        check(self.L.arcos_dump(self.h, self.ids[gid], set, KINDS[what], s, str(path).encode(), 1))

    def load(self, path, gid: int = 0, what: str = "dens", s: int = 0, set: int = SET_GRID):
        """Load a dump written by ``dump`` into the interior (ghosts kept)."""
        check(self.L.arcos_dump(self.h, self.ids[gid], set, KINDS[what], s, str(path).encode(), 0))

    def set_field(self, gid: int, er, ez, etheta=None, set: int = SET_GRID):
        arrs = [None if x is None else np.ascontiguousarray(x, dtype=np.float64) for x in (er, ez, etheta)]
        ptrs = [None if x is None else _dp(x) for x in arrs]
        check(self.L.arcos_set_field(self.h, self.ids[gid], set, *ptrs))

    def field_post(self, set: int = SET_GRID):
        check(self.L.arcos_field_post(self.h, set))

    def set_fixed_field(self, fields: Sequence):
        """Fixed field solve output for every grid: ``fields[gid] = (er, ez,
        etheta)`` (None entries are zero).  Written to both storage sets."""
        for st in (SET_GRID, SET_INTER):
            for gid, f in enumerate(fields):
                self.set_field(gid, *f, set=st)
            self.field_post(st)

    def set_family_field(self, fam: int, Ex: float, Ey: float, Ez: float):
        check(self.L.arcos_set_family_field(self.h, fam, Ex, Ey, Ez))

    def set_field_callback(self, fn: Callable[[int, np.ndarray], tuple]):
        """Field solve in the loop: ``fn(stage, charge) -> (er, ez, etheta)`` on
        the root grid, all in rz layout (the pois_solve_a seam, poisson.c:763)."""
        shape = self.specs[0].shape
        n = int(np.prod(shape))

        def cb(user, stage, ch, er, ez, et):
            try:
                charge = np.ctypeslib.as_array(ch, shape=(n,)).reshape(shape).copy()
                fer, fez, fet = fn(stage, charge)
                for src, dst in ((fer, er), (fez, ez), (fet, et)):
                    out = np.ctypeslib.as_array(dst, shape=(n,))
                    out[:] = 0.0 if src is None else np.asarray(src, dtype=np.float64).reshape(-1)
                return 0
            except Exception:   # a Python exception must not unwind through C
                import traceback
                traceback.print_exc()
                return 1

        self._field_cb = FIELD_FN(cb)
        check(self.L.arcos_set_field_fn(self.h, self._field_cb, None))

    def set_photo(self, model=None):
        """Photoionization of ``model`` (default: the tree's own) on the device:
        its photo terms (file order), source and receiving species
        (photo_calc, src/photo.c:313-345); no terms switches it off."""
        m = model if model is not None else self.model
        n = len(m.photo)
        A = np.array([t.A for t in m.photo] or [0.0], dtype=np.float64)
        lam = np.array([t.lam for t in m.photo] or [0.0], dtype=np.float64)
        check(self.L.arcos_set_photo(self.h, n, _dp(A), _dp(lam), max(m.photo_source, 0),
                                     m.photo_electrons, max(m.photo_ions, 0)))

    def set_field_poisson(self, on: bool = True):
        """Solve the field of every stage on the device (pois_solve_a,
        poisson.c:763, one grid; on a 3-D grid by theta modes, cdr.c:532-580):
        no host round trip per stage."""
        check(self.L.arcos_set_field_poisson(self.h, 1 if on else 0))

    def solve_field(self, set: int = SET_GRID):
        """One device field solve of ``set`` from its current charge."""
        check(self.L.arcos_solve_field(self.h, set))

    # ---- reference entry points ----
    def _call(self, name: str, set: int):
        check(getattr(self.L, name)(self.h, set))
        check(self.L.arcos_sync(self.h))

    def cdr_nonegative_r(self, set=SET_GRID): self._call("arcos_cdr_nonegative_r", set)
    def cdr_set_ext_bnd_r(self, set=SET_GRID): self._call("arcos_cdr_set_ext_bnd_r", set)
    def cdr_set_periodic_r(self, set=SET_GRID): self._call("arcos_cdr_set_periodic_r", set)
    def cdr_restrict_r(self, set=SET_GRID): self._call("arcos_cdr_restrict_r", set)
    def cdr_set_bnd_r(self, set=SET_GRID): self._call("arcos_cdr_set_bnd_r", set)
    def cdr_match_r(self, set=SET_GRID): self._call("arcos_cdr_match_r", set)
    def prepare_grid(self, set=SET_GRID): self._call("arcos_prepare_grid", set)
    def cdr_add_ext_field_r(self, set=SET_GRID): self._call("arcos_cdr_add_ext_field_r", set)
    def cdr_calc_eabs_r(self, set=SET_GRID): self._call("arcos_cdr_calc_eabs_r", set)
    def cdr_calc_charge_r(self, set=SET_GRID): self._call("arcos_cdr_calc_charge_r", set)

    def cdr_refine(self, gid: int, threshold_eabs: float, level_eabs: int, threshold_charge: float,
                   threshold_dens: float, threshold_edge: float, brick_dr: int = 8, brick_dz: int = 8,
                   max_level: int = 4, contains_edge: bool = False) -> List[tuple]:
        """cdr_refine (src/cdr.c:1630-1682) of grid ``gid``: the children
        refine_in would create, in creation order, as (r0, z0, r1, z1,
        contains_edge) in child-level coordinates.  Refine a family's root
        before its other grids (they inherit its maxima)."""
        rp = RefineParams(threshold_eabs, level_eabs, threshold_charge, threshold_dens,
                          threshold_edge, brick_dr, brick_dz, max_level)
        cap = 64
        while True:
            buf = (C.c_int * (5 * cap))()
            n = C.c_int(0)
            rc = self.L.arcos_cdr_refine(self.h, self.ids[gid], C.byref(rp), 1 if contains_edge else 0,
                                         buf, cap, C.byref(n))
            if rc != 0 and n.value > cap:
                cap = n.value
                continue
            check(rc)
            return [tuple(buf[5 * i: 5 * i + 5]) for i in range(n.value)]
    def react_apply_all(self, set=SET_GRID): self._call("arcos_react_apply_all", set)
    def cdr_advect_diffu_r(self, set=SET_GRID): self._call("arcos_cdr_advect_diffu_r", set)
    def cdr_calc_d_dens(self, set=SET_GRID): self._call("arcos_cdr_calc_d_dens", set)

    def cdr_courant(self, set=SET_GRID) -> float:
        h = C.c_double(0.0)
        check(self.L.arcos_cdr_courant(self.h, set, C.byref(h)))
        return h.value

    def cdr_update(self, h: float):
        check(self.L.arcos_cdr_update(self.h, h))
        check(self.L.arcos_sync(self.h))

    def cdr_rk2_update(self, h: float):
        check(self.L.arcos_cdr_rk2_update(self.h, h))
        check(self.L.arcos_sync(self.h))

    def cdr_rk2(self, h: float, t: float = 0.0) -> float:
        hu = C.c_double(0.0)
        check(self.L.arcos_cdr_rk2(self.h, h, t, C.byref(hu)))
        return hu.value

    def run(self, nsteps: int, h: float) -> np.ndarray:
        """``nsteps`` steps of cdr_rk2 for every family; returns dt[fam, step]."""
        nfam = sum(1 for s in self.specs if s.parent < 0)
        dts = np.zeros((nfam, max(nsteps, 1)))
        check(self.L.arcos_run(self.h, nsteps, h, _dp(dts)))
        return dts[:, :nsteps]

    def family_state(self, fam: int = 0):
        st, h, e = C.c_int(0), C.c_double(0), C.c_int(0)
        check(self.L.arcos_family_state(self.h, fam, C.byref(st), C.byref(h), C.byref(e)))
        return st.value, h.value, e.value

    # ---- model parameters after commit ----
    def set_species_mass(self, s: int, mass: float):
        check(self.L.arcos_set_species_mass(self.h, s, mass))

    def set_diffusion(self, diffusion_coeff: float):
        check(self.L.arcos_set_diffusion(self.h, diffusion_coeff))

    def set_table_values(self, reaction: int, values, underflow: float, overflow: float):
        v = np.ascontiguousarray(values, dtype=np.float64)
        check(self.L.arcos_set_table_values(self.h, reaction, _dp(v), underflow, overflow))

    def set_tma(self, on: bool):
        check(self.L.arcos_set_tma(self.h, 1 if on else 0))

    def set_exact(self, on: bool):
        check(self.L.arcos_set_exact(self.h, 1 if on else 0))

    def set_tile(self, cfg: int):
        check(self.L.arcos_set_tile(self.h, cfg))

    @property
    def num_items(self) -> int:
        return self.L.arcos_num_items(self.h)

    def device_bytes(self) -> int:
        n = C.c_size_t(0)
        check(self.L.arcos_device_bytes(self.h, C.byref(n)))
        return n.value


def cdr_advect_vec(mass: float, charge: float, dens: np.ndarray, d_dens: np.ndarray,
                   er: np.ndarray, ez: np.ndarray, diffusion_coeff: float, dr: float,
                   dz: float, r0: int, r1: int, z0: int, z1: int) -> None:
    """The narrow seam with the reference wrapper's argument meaning
    (arcos_f90/src/cdr_advect_diffu_wrap.c:25-41); updates ``d_dens`` in place."""
    L = lib()
    for a in (dens, d_dens, er, ez):
        assert a.dtype == np.float64 and a.flags.c_contiguous
    L.arcos_cdr_advect_vec(mass, charge, _dp(dens), _dp(d_dens), _dp(er), er.size, _dp(ez),
                           ez.size, diffusion_coeff, dr, dz, 0, r0, r1, z0, z1)
