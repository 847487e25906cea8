"""ctypes binding of ``lib/libvsdmo.so`` (the C ABI declared in ``include/vsdmo.h``).

The library is the only compute path: importing this module fails loudly when the shared
object is missing, and every call raises ``VSDMOError`` on a non-zero status. There is no
CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("VSDMO_LIB", os.path.join(HERE, "lib", "libvsdmo.so"))

OK, E_ARG, E_CUDA, E_NONMANIFOLD, E_VALENCE, E_MONOTONE, E_TIMEOUT, E_NAN, E_NOMEM, E_UNSUPPORTED, E_IO = range(11)
FMT_AUTO, FMT_OFF, FMT_TETGEN, FMT_MEDIT = range(4)
TRI, QUAD, TET, HEX = 0, 1, 2, 3
HOST, DEVICE = 0, 1

# every entry point include/vsdmo.h declares (checked by the CPU symbol test)
EXPORTED = [
    "vsdmo_version", "vsdmo_last_error", "vsdmo_status_string", "vsdmo_params_default",
    "vsdmo_mesh_create", "vsdmo_mesh_destroy", "vsdmo_mesh_info", "vsdmo_mesh_array_len",
    "vsdmo_mesh_array", "vsdmo_mesh_permutation", "vsdmo_mesh_get_positions",
    "vsdmo_mesh_set_positions", "vsdmo_mesh_sync", "vsdmo_opt_create", "vsdmo_opt_destroy",
    "vsdmo_opt_iterate", "vsdmo_opt_restart", "vsdmo_opt_optimize", "vsdmo_opt_is_done", "vsdmo_opt_iterations_done",
    "vsdmo_opt_get_quality", "vsdmo_opt_find_min_quality", "vsdmo_opt_element_qualities",
    "vsdmo_opt_quality_histogram", "vsdmo_opt_display_quality", "vsdmo_opt_history",
    "vsdmo_opt_run_color", "vsdmo_opt_launches_per_iteration", "vsdmo_opt_surface_state",
    "vsdmo_quality_reduce_noalloc", "vsdmo_model_num_params", "vsdmo_model_create", "vsdmo_model_destroy",
    "vsdmo_model_get_params", "vsdmo_model_set_params", "vsdmo_model_forward", "vsdmo_model_gradients",
    "vsdmo_model_train", "vsdmo_opt_collect_pairs", "vsdmo_opt_set_model", "vsdmo_opt_learned_counters",
    "vsdmo_debug_gemm_bf16", "vsdmo_debug_set_wait_limit_ns", "vsdmo_opt_proposals", "vsdmo_opt_set_proposal_schedule",
    "vsdmo_batch_create", "vsdmo_batch_destroy", "vsdmo_batch_iterate", "vsdmo_batch_iterate_async",
    "vsdmo_batch_sync", "vsdmo_batch_restart", "vsdmo_batch_stats", "vsdmo_batch_get_positions",
    "vsdmo_batch_set_positions", "vsdmo_batch_get_config", "vsdmo_batch_set_config", "vsdmo_batch_autotune",
    "vsdmo_batch_info", "vsdmo_batch_mesh_info",
    "vsdmo_file_read", "vsdmo_file_write", "vsdmo_mesh_create_from_file", "vsdmo_mesh_write_file",
    "vsdmo_mesh_create_surface", "vsdmo_opt_local_surface_points", "vsdmo_opt_estimate_surface_points",
    "vsdmo_opt_feature_state",
]


class VSDMOError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"vsdmo status {status}: {msg}")
        self.status = status


class Params(C.Structure):
    _fields_ = [("quality", C.c_int), ("grid_scale", C.c_float), ("n_iter", C.c_int),
                ("grid_n", C.c_int), ("depth", C.c_int), ("fix_boundary", C.c_int),
                ("flat", C.c_int), ("use_graph", C.c_int), ("check_monotone", C.c_int),
                ("active_set", C.c_int), ("fit_ring", C.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"CUDA library {LIB_PATH} is missing; build it with "
                          "`python volumesurfacediscretemeshoptimization_b200/build.py`")
    L = C.CDLL(LIB_PATH)
    P, I, U, F = C.c_void_p, C.c_int, C.c_uint32, C.c_float
    S = C.c_int  # vsdmo_status
    L.vsdmo_version.restype = C.c_char_p
    L.vsdmo_last_error.restype = C.c_char_p
    L.vsdmo_status_string.restype = C.c_char_p
    L.vsdmo_status_string.argtypes = [I]
    L.vsdmo_params_default.restype = S
    L.vsdmo_params_default.argtypes = [I, C.POINTER(Params)]
    L.vsdmo_mesh_create.restype = S
    L.vsdmo_mesh_create.argtypes = [I, P, I, P, I, I, U, P, C.POINTER(P)]
    L.vsdmo_mesh_destroy.argtypes = [P]
    L.vsdmo_mesh_destroy.restype = None
    L.vsdmo_mesh_info.argtypes = [P, I]
    L.vsdmo_mesh_array_len.restype = C.c_long
    L.vsdmo_mesh_array_len.argtypes = [P, I]
    L.vsdmo_mesh_array.restype = S
    L.vsdmo_mesh_array.argtypes = [P, I, P]
    L.vsdmo_mesh_permutation.restype = S
    L.vsdmo_mesh_permutation.argtypes = [P, P]
    L.vsdmo_mesh_get_positions.restype = S
    L.vsdmo_mesh_get_positions.argtypes = [P, P, I, I]
    L.vsdmo_mesh_set_positions.restype = S
    L.vsdmo_mesh_set_positions.argtypes = [P, P, I, I]
    L.vsdmo_mesh_sync.restype = S
    L.vsdmo_mesh_sync.argtypes = [P]
    L.vsdmo_opt_create.restype = S
    L.vsdmo_opt_create.argtypes = [P, C.POINTER(Params), C.POINTER(P)]
    L.vsdmo_opt_destroy.argtypes = [P]
    L.vsdmo_opt_destroy.restype = None
    L.vsdmo_opt_iterate.restype = S
    L.vsdmo_opt_iterate.argtypes = [P, I]
    L.vsdmo_opt_restart.restype = S
    L.vsdmo_opt_restart.argtypes = [P]
    L.vsdmo_opt_optimize.restype = S
    L.vsdmo_opt_optimize.argtypes = [P]
    L.vsdmo_opt_is_done.argtypes = [P]
    L.vsdmo_opt_iterations_done.argtypes = [P]
    L.vsdmo_opt_launches_per_iteration.argtypes = [P]
    L.vsdmo_opt_surface_state.argtypes = [P, P, P, P]
    L.vsdmo_opt_get_quality.restype = S
    L.vsdmo_opt_get_quality.argtypes = [P, C.POINTER(F)]
    L.vsdmo_opt_find_min_quality.restype = S
    L.vsdmo_opt_find_min_quality.argtypes = [P, C.POINTER(F), C.POINTER(C.c_double)]
    L.vsdmo_opt_element_qualities.restype = S
    L.vsdmo_opt_element_qualities.argtypes = [P, P, I]
    L.vsdmo_opt_quality_histogram.restype = S
    L.vsdmo_opt_quality_histogram.argtypes = [P, P, I]
    L.vsdmo_opt_display_quality.restype = S
    L.vsdmo_opt_display_quality.argtypes = [P, I]
    L.vsdmo_opt_history.restype = S
    L.vsdmo_opt_history.argtypes = [P, P, P, I, C.POINTER(I)]
    L.vsdmo_opt_run_color.restype = S
    L.vsdmo_opt_run_color.argtypes = [P, I]
    L.vsdmo_quality_reduce_noalloc.restype = S
    L.vsdmo_quality_reduce_noalloc.argtypes = [I, I, P, I, P, I, F, P, P, P, P]
    Lg, U64 = C.c_long, C.c_uint64
    L.vsdmo_model_num_params.argtypes = []
    L.vsdmo_model_create.restype = S
    L.vsdmo_model_create.argtypes = [U64, P, C.POINTER(P)]
    L.vsdmo_model_destroy.restype = None
    L.vsdmo_model_destroy.argtypes = [P]
    L.vsdmo_model_get_params.restype = S
    L.vsdmo_model_get_params.argtypes = [P, P]
    L.vsdmo_model_set_params.restype = S
    L.vsdmo_model_set_params.argtypes = [P, P]
    L.vsdmo_model_forward.restype = S
    L.vsdmo_model_forward.argtypes = [P, P, Lg, P, I]
    L.vsdmo_model_gradients.restype = S
    L.vsdmo_model_gradients.argtypes = [P, P, P, I, C.POINTER(F), P]
    L.vsdmo_model_train.restype = S
    L.vsdmo_model_train.argtypes = [P, P, P, Lg, I, I, I, F, U64, P]
    L.vsdmo_opt_collect_pairs.restype = S
    L.vsdmo_opt_collect_pairs.argtypes = [P, I, P, P, Lg, C.POINTER(Lg)]
    L.vsdmo_opt_set_model.restype = S
    L.vsdmo_opt_set_model.argtypes = [P, P, I, I, F]
    L.vsdmo_opt_learned_counters.restype = S
    L.vsdmo_opt_learned_counters.argtypes = [P, P]
    L.vsdmo_opt_set_proposal_schedule.restype = S
    L.vsdmo_opt_set_proposal_schedule.argtypes = [P, I]
    L.vsdmo_opt_proposals.restype = S
    L.vsdmo_opt_proposals.argtypes = [P, I, P]
    L.vsdmo_debug_gemm_bf16.restype = S
    L.vsdmo_debug_gemm_bf16.argtypes = [P, P, I, I, I, P]
    L.vsdmo_debug_set_wait_limit_ns.restype = S
    L.vsdmo_debug_set_wait_limit_ns.argtypes = [C.c_int64]
    L.vsdmo_batch_create.restype = S
    L.vsdmo_batch_create.argtypes = [I, P, P, P, P, P, I, U, P, C.POINTER(P)]
    L.vsdmo_batch_destroy.restype = None
    L.vsdmo_batch_destroy.argtypes = [P]
    for name in ("vsdmo_batch_iterate", "vsdmo_batch_iterate_async"):
        getattr(L, name).restype = S
        getattr(L, name).argtypes = [P, I]
    for name in ("vsdmo_batch_sync", "vsdmo_batch_restart"):
        getattr(L, name).restype = S
        getattr(L, name).argtypes = [P]
    L.vsdmo_batch_stats.restype = S
    L.vsdmo_batch_stats.argtypes = [P, I, P, P, P]
    L.vsdmo_batch_get_positions.restype = S
    L.vsdmo_batch_get_positions.argtypes = [P, P, I]
    L.vsdmo_batch_set_positions.restype = S
    L.vsdmo_batch_set_positions.argtypes = [P, P, I]
    L.vsdmo_batch_get_config.restype = S
    L.vsdmo_batch_get_config.argtypes = [P, P, P, P]
    L.vsdmo_batch_set_config.restype = S
    L.vsdmo_batch_set_config.argtypes = [P, P, P, P]
    L.vsdmo_batch_autotune.restype = S
    L.vsdmo_batch_autotune.argtypes = [P, I, C.c_char_p, I]
    L.vsdmo_batch_info.restype = C.c_long
    L.vsdmo_batch_info.argtypes = [P, I]
    L.vsdmo_file_read.restype = S
    L.vsdmo_file_read.argtypes = [C.c_char_p, I, C.POINTER(I), C.POINTER(I), C.POINTER(I), P, P]
    L.vsdmo_file_write.restype = S
    L.vsdmo_file_write.argtypes = [C.c_char_p, I, I, P, I, P, I]
    L.vsdmo_mesh_create_from_file.restype = S
    L.vsdmo_mesh_create_from_file.argtypes = [C.c_char_p, I, U, P, C.POINTER(P)]
    L.vsdmo_mesh_write_file.restype = S
    L.vsdmo_mesh_write_file.argtypes = [P, C.c_char_p, I]
    L.vsdmo_mesh_create_surface.restype = S
    L.vsdmo_mesh_create_surface.argtypes = [P, U, P, C.POINTER(P)]
    L.vsdmo_opt_feature_state.restype = S
    L.vsdmo_opt_feature_state.argtypes = [P, P, P, P, P, P, P, C.POINTER(I)]
    L.vsdmo_opt_local_surface_points.restype = S
    L.vsdmo_opt_local_surface_points.argtypes = [P, I, I, I, P, I, I]
    L.vsdmo_opt_estimate_surface_points.restype = S
    L.vsdmo_opt_estimate_surface_points.argtypes = [P, I, I, I, P, I]
    L.vsdmo_batch_mesh_info.restype = S
    L.vsdmo_batch_mesh_info.argtypes = [P, I, P]
    _lib = L
    return L


def check(status):
    if status != OK:
        msg = lib().vsdmo_last_error().decode(errors="replace")
        raise VSDMOError(status, msg or lib().vsdmo_status_string(status).decode())
