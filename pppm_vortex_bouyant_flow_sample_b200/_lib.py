"""ctypes binding of libpppm_b200.so (the C ABI declared in include/pppm.h).

Loading fails loudly: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

from . import _build

PPPM_OK = 0
STATUS_NAMES = {0: "PPPM_OK", 1: "PPPM_ERR_INVALID", 2: "PPPM_ERR_CUDA", 3: "PPPM_ERR_OOM",
                4: "PPPM_ERR_STATE", 5: "PPPM_ERR_DOMAIN"}
DOMAIN_BBOX3X, DOMAIN_FIXED = 0, 1
MG_REFERENCE, MG_CONVERGED = 0, 1
GRID_VORT, GRID_PSI, GRID_FAR = 0, 1, 2

# Every symbol include/pppm.h declares; tests check the library exports them.
EXPORTED = (
    "pppm_last_error", "pppm_version", "pppm_params_default", "pppm_scene_create",
    "pppm_scene_destroy", "pppm_scene_set_stream", "pppm_scene_get_params", "pppm_set_vortices",
    "pppm_build_far_field", "pppm_eval", "pppm_eval_f32", "pppm_solve_host", "pppm_get_domain",
    "pppm_get_cell_tables", "pppm_get_sorted_index", "pppm_get_sorted_vortices", "pppm_get_grid",
    "pppm_get_stats", "pppm_count_pairs", "pppm_mg_create", "pppm_mg_destroy",
    "pppm_mg_full_multigrid", "pppm_hasher_create", "pppm_hasher_destroy", "pppm_hasher_run",
    "pppm_hasher_tables", "pppm_hasher_reorder", "pppm_hasher_deorder", "pppm_direct_sum_fp64",
    "pppm_scene_set_profiling", "pppm_stage_name", "pppm_get_stage_times", "pppm_kernel_launches",
    "pppm_spatial_hash_noalloc", "pppm_advect_euler", "pppm_advect_rk2", "pppm_batch_run",
    "pppm_server_create", "pppm_server_destroy", "pppm_server_add_scene", "pppm_server_submit",
    "pppm_server_wait", "pppm_server_read_positions", "pppm_server_stats",
    "pppm_frame_path", "pppm_write_frame", "pppm_read_frame", "pppm_vortex_step",
    "pppm_baroclinic", "pppm_get_density", "pppm_write_sgi", "pppm_renderer_create", "pppm_renderer_destroy",
    "pppm_render_shadows", "pppm_render_shadow_map", "pppm_render_smoke", "pppm_potential_create",
    "pppm_potential_destroy", "pppm_potential_set_masses", "pppm_potential_build", "pppm_potential_eval_gradient",
    "pppm_potential_eval_scalar", "pppm_potential_dphidn", "pppm_potential_grids", "pppm_potential_eval_gradient3",
    "pppm_debug_fail_allocation", "pppm_mg_vcycle", "pppm_mg_levels", "pppm_params_accurate",
    "pppm_get_smoothing", "pppm_tuning_report",
)
REQ_EVAL, REQ_ADVANCE = 0, 1
NOALLOC_MAX_PARTICLES = 1048576  # PPPM_NOALLOC_MAX_PARTICLES in include/pppm.h
STAGES = ("domain", "vort_sort", "cells_reorder", "p2m", "multigrid", "farfield", "eval_sort", "eval",
          "segments", "seg_to_blob", "rehash", "gaussian_smooth")


class PppmParams(C.Structure):
    _fields_ = [
        ("n", C.c_uint32),
        ("K", C.c_int32),
        ("a", C.c_double),
        ("domain_mode", C.c_int32),
        ("fixed_origin", C.c_double * 3),
        ("fixed_length", C.c_double),
        ("mg_mode", C.c_int32),
        ("mg_tol", C.c_double),
        ("mg_max_cycles", C.c_int32),
        ("a_cells", C.c_double),
    ]


class PppmBatchItem(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("N", C.c_uint32), ("pos4_dev", C.c_void_p), ("ax_dev", C.c_void_p),
                ("ay_dev", C.c_void_p), ("az_dev", C.c_void_p), ("M", C.c_uint32), ("eval_a4_dev", C.c_void_p),
                ("eval_b4_dev", C.c_void_p), ("is_segment", C.c_int), ("u_dev", C.c_void_p), ("v_dev", C.c_void_p),
                ("w_dev", C.c_void_p)]


class PppmServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("slots", C.c_uint32)]


class PppmRequestInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("submit_s", C.c_double), ("start_s", C.c_double), ("end_s", C.c_double)]


class PppmError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_lib = None
vp = C.c_void_p
u32 = C.c_uint32
i32 = C.c_int32


def library_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load the library (building it in-tree first if it is missing or stale)."""
    global _lib
    if _lib is not None:
        return _lib
    if build_if_missing and not _build.up_to_date():
        _build.build()
    path = library_path()
    if not os.path.exists(path):
        raise ImportError(f"libpppm_b200.so not found at {path}; run __graft_entry__.build()")
    L = C.CDLL(path)
    st = C.c_int
    sig = {
        "pppm_last_error": (C.c_char_p, []),
        "pppm_version": (C.c_char_p, []),
        "pppm_params_default": (st, [C.POINTER(PppmParams)]),
        "pppm_scene_create": (st, [C.POINTER(PppmParams), u32, u32, vp, C.POINTER(vp)]),
        "pppm_scene_destroy": (st, [vp]),
        "pppm_scene_set_stream": (st, [vp, vp]),
        "pppm_scene_get_params": (st, [vp, C.POINTER(PppmParams)]),
        "pppm_set_vortices": (st, [vp, u32, vp, vp, vp, vp]),
        "pppm_build_far_field": (st, [vp]),
        "pppm_eval": (st, [vp, u32, vp, vp, C.c_int, vp, vp, vp]),
        "pppm_eval_f32": (st, [vp, u32, vp, vp, C.c_int, vp]),
        "pppm_solve_host": (st, [vp, u32, vp, vp, vp, vp, u32, vp, vp, C.c_int, vp, vp, vp]),
        "pppm_get_domain": (st, [vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]),
        "pppm_get_cell_tables": (st, [vp, C.POINTER(vp), C.POINTER(vp)]),
        "pppm_get_sorted_index": (st, [vp, C.POINTER(vp), C.POINTER(vp)]),
        "pppm_get_sorted_vortices": (st, [vp, vp, vp, vp, vp]),
        "pppm_get_grid": (st, [vp, C.c_int, C.POINTER(vp)]),
        "pppm_get_stats": (st, [vp, C.POINTER(C.c_uint64), C.POINTER(i32), C.POINTER(C.c_double)]),
        "pppm_count_pairs": (st, [vp, u32, vp, C.POINTER(C.c_uint64)]),
        "pppm_mg_create": (st, [u32, vp, C.POINTER(vp)]),
        "pppm_mg_destroy": (st, [vp]),
        "pppm_mg_full_multigrid": (st, [vp, vp, vp, C.c_int, C.c_double, C.c_int, C.POINTER(C.c_double)]),
        "pppm_tuning_report": (st, [C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
        "pppm_params_accurate": (st, [C.POINTER(PppmParams)]),
        "pppm_get_smoothing": (st, [vp, C.POINTER(C.c_double)]),
        "pppm_mg_vcycle": (st, [vp, vp, vp, C.c_int]),
        "pppm_mg_levels": (st, [vp, C.POINTER(C.c_int), C.POINTER(u32), C.c_int]),
        "pppm_hasher_create": (st, [u32, u32, vp, C.POINTER(vp)]),
        "pppm_hasher_destroy": (st, [vp]),
        "pppm_hasher_run": (st, [vp, u32, vp, C.c_float, C.POINTER(C.c_float)]),
        "pppm_hasher_tables": (st, [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]),
        "pppm_hasher_reorder": (st, [vp, u32, vp, vp, u32, u32]),
        "pppm_hasher_deorder": (st, [vp, u32, vp, vp, u32, u32]),
        "pppm_direct_sum_fp64": (st, [u32, vp, vp, vp, vp, u32, vp, vp, C.c_int, C.c_double, vp, vp, vp, vp]),
        "pppm_scene_set_profiling": (st, [vp, C.c_int]),
        "pppm_stage_name": (C.c_char_p, [C.c_int]),
        "pppm_get_stage_times": (st, [vp, C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_int)]),
        "pppm_kernel_launches": (C.c_uint64, []),
        "pppm_debug_fail_allocation": (st, [C.c_int64]),
        "pppm_spatial_hash_noalloc": (st, [u32, vp, u32, C.c_float, C.POINTER(C.c_float), vp, vp, vp, vp, vp]),
        "pppm_advect_euler": (st, [vp, u32, vp, vp, vp, vp, C.c_double]),
        "pppm_advect_rk2": (st, [vp, u32, vp, vp, vp, vp, C.c_double]),
        "pppm_vortex_step": (st, [vp, u32, vp, vp, vp, vp, C.c_double, C.c_double, C.c_double, vp, vp, u32, vp,
                                  vp, vp, vp]),
        "pppm_baroclinic": (st, [vp, u32, vp, vp, u32, vp, vp, vp, vp, C.c_double]),
        "pppm_write_sgi": (st, [C.c_char_p, u32, u32, C.c_int, vp, C.c_int]),
        "pppm_potential_create": (st, [u32, C.c_int, u32, u32, vp, C.POINTER(vp)]),
        "pppm_potential_destroy": (st, [vp]),
        "pppm_potential_set_masses": (st, [vp, u32, vp, vp]),
        "pppm_potential_build": (st, [vp, C.c_int]),
        "pppm_potential_eval_gradient": (st, [vp, u32, vp, vp, vp, vp]),
        "pppm_potential_eval_scalar": (st, [vp, u32, vp, vp]),
        "pppm_potential_eval_gradient3": (st, [vp, u32, vp, vp]),
        "pppm_potential_dphidn": (st, [vp, u32, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
        "pppm_potential_grids": (st, [vp, C.POINTER(C.c_double), C.POINTER(vp), C.POINTER(vp), C.POINTER(vp),
                                      C.POINTER(vp), C.POINTER(C.c_double)]),
        "pppm_renderer_create": (st, [vp, C.POINTER(vp)]),
        "pppm_renderer_destroy": (st, [vp]),
        "pppm_render_shadows": (st, [vp, u32, vp, vp, C.c_float, C.c_float, C.POINTER(C.c_float), C.c_float, vp,
                                     C.POINTER(u32)]),
        "pppm_render_shadow_map": (st, [vp, C.POINTER(vp), C.POINTER(u32)]),
        "pppm_render_smoke": (st, [vp, u32, vp, vp, vp, vp, C.c_float, C.c_float, vp, C.POINTER(C.c_float),
                                   C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_float, u32, u32, vp]),
        "pppm_get_density": (st, [vp, C.POINTER(u32), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                  C.POINTER(vp), C.POINTER(vp)]),
        "pppm_batch_run": (st, [C.POINTER(PppmBatchItem), u32, vp]),
        "pppm_server_create": (st, [C.POINTER(PppmServerConfig), C.POINTER(vp)]),
        "pppm_server_destroy": (st, [vp]),
        "pppm_server_add_scene": (st, [vp, C.POINTER(PppmParams), u32, vp, vp, vp, vp, C.POINTER(C.c_uint64)]),
        "pppm_server_submit": (st, [vp, C.c_uint64, C.c_int, u32, C.c_double, C.POINTER(C.c_uint64)]),
        "pppm_server_wait": (st, [vp, C.c_uint64, C.c_double, C.POINTER(PppmRequestInfo), vp]),
        "pppm_server_read_positions": (st, [vp, C.c_uint64, vp]),
        "pppm_server_stats": (st, [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
        "pppm_frame_path": (st, [C.c_char_p, C.c_int, C.c_char_p, C.c_size_t]),
        "pppm_write_frame": (st, [C.c_char_p, C.c_int, u32, vp, C.c_int]),
        "pppm_read_frame": (st, [C.c_char_p, vp, u32, C.POINTER(u32)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return _lib


def check(status: int, where: str):
    if status != PPPM_OK:
        msg = load().pppm_last_error().decode(errors="replace")
        raise PppmError(status, where, msg)


def default_params(n: int, **kw) -> PppmParams:
    p = PppmParams()
    check(load().pppm_params_default(C.byref(p)), "pppm_params_default")
    p.n = n
    for k, v in kw.items():
        if k == "fixed_origin":
            p.fixed_origin[:] = list(v)
        else:
            setattr(p, k, v)
    return p
