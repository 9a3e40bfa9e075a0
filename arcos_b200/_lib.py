"""Loader for the device library ``libarcos_cdr.so`` (C ABI of
include/arcos_cdr.h).  There is no CPU fallback: every entry point of this
package needs the library and a CUDA device, and raises if either is missing."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libarcos_cdr.so")

DP = C.POINTER(C.c_double)
VP = C.c_void_p

ARCOS_OK = 0
ERRORS = {1: "ARCOS_ERR_ARG", 2: "ARCOS_ERR_CUDA", 3: "ARCOS_ERR_NAN", 4: "ARCOS_ERR_SMALL_DT",
          5: "ARCOS_ERR_TIMEOUT", 6: "ARCOS_ERR_NOMEM", 7: "ARCOS_ERR_STATE"}

MAX_SPECIES = 16


class ArcosParams(C.Structure):
    """``arcos_params`` of include/arcos_cdr.h."""
    _fields_ = [("no_species", C.c_int), ("charge", C.c_double * MAX_SPECIES),
                ("mass", C.c_double * MAX_SPECIES), ("diffusion_coeff", C.c_double),
                ("nu_a", C.c_double), ("nu_d", C.c_double), ("nu_rt", C.c_double),
                ("warn_min_timestep", C.c_double), ("cdr_bnd_bottom", C.c_int),
                ("cdr_bnd_top", C.c_int), ("cdr_bnd_right", C.c_int), ("E_x", C.c_double),
                ("E_y", C.c_double), ("E_z", C.c_double), ("z_cutoff", C.c_double),
                ("L_r", C.c_double), ("L_z", C.c_double), ("gridpoints_r", C.c_int),
                ("gridpoints_z", C.c_int), ("max_ntheta", C.c_int), ("max_levels", C.c_int),
                ("extra_pois_levels", C.c_int), ("per_plane", C.c_int)]


class RefineParams(C.Structure):
    """``arcos_refine_params`` of include/arcos_cdr.h (the refinement
    parameters of the reference's src/parameters.h)."""
    _fields_ = [("threshold_eabs", C.c_double), ("level_eabs", C.c_int),
                ("threshold_charge", C.c_double), ("threshold_dens", C.c_double),
                ("threshold_edge", C.c_double), ("brick_dr", C.c_int), ("brick_dz", C.c_int),
                ("max_level", C.c_int)]


FIELD_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, DP, DP, DP, DP)

_lib = None


class ArcosError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"device library missing: {LIB_PATH}; run __graft_entry__.build()")
    L = C.CDLL(LIB_PATH)
    L.arcos_last_error.restype = C.c_char_p
    L.arcos_create.argtypes = [C.POINTER(ArcosParams), C.POINTER(VP)]
    for name in ("arcos_destroy", "arcos_commit", "arcos_sync", "arcos_num_items"):
        getattr(L, name).argtypes = [VP]
    L.arcos_set_stream.argtypes = [VP, VP]
    L.arcos_add_reaction.argtypes = [VP, C.c_int, C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_int),
                                     C.c_double, C.c_double, C.c_int, C.c_double, C.c_double, DP]
    L.arcos_grid_new.argtypes = [VP, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                 C.c_int, C.POINTER(C.c_int)]
    L.arcos_device_bytes.argtypes = [VP, C.POINTER(C.c_size_t)]
    L.arcos_upload.argtypes = [VP, C.c_int, C.c_int, C.c_int, C.c_int, DP]
    L.arcos_download.argtypes = [VP, C.c_int, C.c_int, C.c_int, C.c_int, DP]
    L.arcos_set_field.argtypes = [VP, C.c_int, C.c_int, DP, DP, DP]
    L.arcos_set_field_fn.argtypes = [VP, FIELD_FN, VP]
    L.arcos_set_field_poisson.argtypes = [VP, C.c_int]
    L.arcos_set_photo.argtypes = [VP, C.c_int, DP, DP, C.c_int, C.c_int, C.c_int]
    L.arcos_set_vjp_form.argtypes = [VP, C.c_int]
    L.arcos_dump.argtypes = [VP, C.c_int, C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_int]
    L.arcos_solve_field.argtypes = [VP, C.c_int]
    for name in ("arcos_cdr_nonegative_r", "arcos_cdr_set_ext_bnd_r", "arcos_cdr_set_periodic_r",
                 "arcos_cdr_restrict_r", "arcos_cdr_set_bnd_r", "arcos_cdr_match_r",
                 "arcos_prepare_grid", "arcos_cdr_add_ext_field_r", "arcos_cdr_calc_eabs_r",
                 "arcos_cdr_calc_charge_r", "arcos_react_apply_all", "arcos_cdr_advect_diffu_r",
                 "arcos_cdr_calc_d_dens", "arcos_field_post", "arcos_set_per_patch",
                 "arcos_set_tile", "arcos_set_exact", "arcos_set_tma", "arcos_run_enqueue"):
        getattr(L, name).argtypes = [VP, C.c_int]
    L.arcos_get_tile.argtypes = [VP]
    L.arcos_cdr_courant.argtypes = [VP, C.c_int, DP]
    L.arcos_cdr_update.argtypes = [VP, C.c_double]
    L.arcos_cdr_rk2_update.argtypes = [VP, C.c_double]
    L.arcos_cdr_rk2.argtypes = [VP, C.c_double, C.c_double, DP]
    L.arcos_run.argtypes = [VP, C.c_int, C.c_double, DP]
    L.arcos_run_prepare.argtypes = [VP, C.c_double]
    L.arcos_enqueue_stage.argtypes = [VP, C.c_int, C.c_int]
    L.arcos_set_family_field.argtypes = [VP, C.c_int, C.c_double, C.c_double, C.c_double]
    L.arcos_family_state.argtypes = [VP, C.c_int, C.POINTER(C.c_int), DP, C.POINTER(C.c_int)]
    L.arcos_cdr_advect_vec.argtypes = [C.c_double, C.c_double, DP, DP, DP, C.c_int, DP, C.c_int,
                                       C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                       C.c_int, C.c_int, C.c_int]
    L.arcos_cdr_advect_vec.restype = None
    L.arcos_cdr_advect_vec_dev.argtypes = [C.c_double, C.c_double, VP, VP, VP, VP, C.c_double,
                                           C.c_double, C.c_double, C.c_int, C.c_int, C.c_int,
                                           C.c_int, VP]
    L.arcos_set_species_mass.argtypes = [VP, C.c_int, C.c_double]
    L.arcos_set_diffusion.argtypes = [VP, C.c_double]
    L.arcos_set_table_values.argtypes = [VP, C.c_int, DP, C.c_double, C.c_double]
    L.arcos_adj_forward.argtypes = [VP, C.c_int, C.c_int, C.c_double, DP, DP]
    L.arcos_adj_set_cotangent.argtypes = [VP, C.c_int, C.c_int, DP]
    L.arcos_adj_get_cotangent.argtypes = [VP, C.c_int, C.c_int, DP]
    L.arcos_adj_backward.argtypes = [VP, DP, DP, DP]
    L.arcos_adj_table_entries.argtypes = [VP]
    L.arcos_adj_table_offset.argtypes = [VP, C.c_int]
    L.arcos_cdr_refine.argtypes = [VP, C.c_int, C.POINTER(RefineParams), C.c_int,
                                   C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_int)]
    _lib = L
    return L


def check(rc: int):
    if rc != ARCOS_OK:
        raise ArcosError(rc, lib().arcos_last_error().decode(errors="replace"))
