"""ctypes declarations of the C ABI in include/jsi_b200.h.

The shared library is loaded from the package directory; there is no
fallback: if libjsi_b200.so is missing or cannot be loaded, every call raises.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libjsi_b200.so"

MAX_ROUNDS = 16
RECORD_SIZE = 18

JSI_OK = 0
STATUS_NAMES = {
    0: "JSI_OK", -1: "JSI_ERR_INVALID", -2: "JSI_ERR_CUDA", -3: "JSI_ERR_NOMEM", -4: "JSI_ERR_CAPACITY",
    -5: "JSI_ERR_SURFACE", -6: "JSI_ERR_TIMEOUT", -7: "JSI_ERR_UNSUPPORTED", -8: "JSI_ERR_NO_DEVICE",
}

PREC_V5_FP32 = 0
PREC_FP64 = 1
PREC_FP32_SCREEN = 2
PRECISIONS = {"v5_fp32": PREC_V5_FP32, "fp64": PREC_FP64, "fp32_screen": PREC_FP32_SCREEN}

# Every symbol include/jsi_b200.h declares.
EXPORTED = [
    "jsi_abi_version", "jsi_status_string", "jsi_last_error", "jsi_create", "jsi_destroy",
    "jsi_surface_upload", "jsi_surface_upload_many", "jsi_host_alloc", "jsi_host_free", "jsi_surface_release", "jsi_surface_release_many",
    "jsi_surface_domains", "jsi_resident_bytes", "jsi_context_stream",
    "jsi_transfer_bytes", "jsi_launch_count", "jsi_kernel_timing", "jsi_kernel_time", "jsi_kernel_units", "jsi_kernel_names",
    "jsi_dist_params_default",
    "jsi_min_distance", "jsi_inter_params_default", "jsi_intersect", "jsi_bounds_params_default",
    "jsi_distance_bounds", "jsi_surface_curvature_bounds", "jsi_curve_params_default", "jsi_intersection_curves", "jsi_eval_grid", "jsi_eval_grid_f64",
    "jsi_eval_grid_noalloc", "jsi_workers", "jsi_submit_distance", "jsi_submit_intersect", "jsi_wait",
    "jsi_queue_depth", "jsi_min_distance_batch", "jsi_submit_distance_batch", "jsi_wait_distance_batch", "jsi_batch_chunk", "jsi_batch_reruns", "jsi_batch_graphs", "jsi_autotune_batch",
    "jsi_query_batch", "jsi_poll_distance_batch",
]


class Config(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("arena_bytes", ctypes.c_ulonglong),
                ("hbm_budget_bytes", ctypes.c_ulonglong)]


class Task(ctypes.Structure):
    _fields_ = [("surface", ctypes.c_int), ("ustart", ctypes.c_float), ("vstart", ctypes.c_float),
                ("ustop", ctypes.c_float), ("vstop", ctypes.c_float), ("nuv", ctypes.c_int), ("side", ctypes.c_int)]


class DistParams(ctypes.Structure):
    _fields_ = [("nuv_refine", ctypes.c_int), ("k", ctypes.c_int), ("rounds", ctypes.c_int),
                ("precision", ctypes.c_int), ("newton", ctypes.c_int)]


class DistResult(ctypes.Structure):
    _fields_ = [("v5_value", ctypes.c_float), ("distance", ctypes.c_double), ("newton_distance", ctypes.c_double),
                ("uv1", ctypes.c_double * 2), ("uv2", ctypes.c_double * 2), ("point1", ctypes.c_double * 3),
                ("point2", ctypes.c_double * 3), ("rounds_run", ctypes.c_int), ("npairs", ctypes.c_int * MAX_ROUNDS),
                ("kth_d2", ctypes.c_double * MAX_ROUNDS), ("pair_tests", ctypes.c_longlong * MAX_ROUNDS),
                ("candidates", ctypes.c_longlong * MAX_ROUNDS), ("trace_pairs", ctypes.POINTER(ctypes.c_int)),
                ("trace_cap", ctypes.c_longlong), ("device_ms", ctypes.c_float),
                ("tile_pairs", ctypes.c_longlong * MAX_ROUNDS), ("tile_pairs_tested", ctypes.c_longlong * MAX_ROUNDS),
                ("supertile_pairs", ctypes.c_longlong * MAX_ROUNDS),
                ("cand_pairs", ctypes.POINTER(ctypes.c_int)), ("cand_d2", ctypes.POINTER(ctypes.c_double)),
                ("cand_cap", ctypes.c_longlong), ("cand_written", ctypes.c_longlong)]


class InterParams(ctypes.Structure):
    _fields_ = [("nuv_refine", ctypes.c_int), ("use_k", ctypes.c_int), ("rounds", ctypes.c_int),
                ("halve_threshold", ctypes.c_int), ("min_nuv", ctypes.c_int), ("precision", ctypes.c_int),
                ("points", ctypes.c_int)]


class InterResult(ctypes.Structure):
    _fields_ = [("rounds_run", ctypes.c_int), ("counts", ctypes.c_longlong * MAX_ROUNDS),
                ("pair_tests", ctypes.c_longlong * MAX_ROUNDS), ("regions1", ctypes.c_longlong * MAX_ROUNDS),
                ("regions2", ctypes.c_longlong * MAX_ROUNDS), ("pad", ctypes.c_double * 2),
                ("trace_pairs", ctypes.POINTER(ctypes.c_int)), ("trace_cap", ctypes.c_longlong),
                ("trace_written", ctypes.c_longlong), ("points", ctypes.POINTER(ctypes.c_double)),
                ("points_cap", ctypes.c_longlong), ("points_written", ctypes.c_longlong),
                ("points_converged", ctypes.c_longlong), ("device_ms", ctypes.c_float),
                ("screen_pairs", ctypes.POINTER(ctypes.c_int)), ("screen_cap", ctypes.c_longlong),
                ("screen_written", ctypes.c_longlong), ("kmax_rechecked", ctypes.c_longlong)]


class CurveParams(ctypes.Structure):
    _fields_ = [("inter", InterParams), ("link_tol", ctypes.c_double)]


class CurveResult(ctypes.Structure):
    _fields_ = [("points_found", ctypes.c_longlong), ("vertices", ctypes.c_longlong), ("curves", ctypes.c_longlong),
                ("link_tol", ctypes.c_double), ("vertex", ctypes.POINTER(ctypes.c_double)),
                ("vertex_cap", ctypes.c_longlong), ("curve_start", ctypes.POINTER(ctypes.c_longlong)),
                ("curve_closed", ctypes.POINTER(ctypes.c_int)), ("curve_cap", ctypes.c_longlong),
                ("device_ms", ctypes.c_float)]


class BoundsParams(ctypes.Structure):
    _fields_ = [("nuv_refine", ctypes.c_int), ("max_rounds", ctypes.c_int), ("rel_tol", ctypes.c_double),
                ("max_pairs", ctypes.c_longlong)]


class BoundsResult(ctypes.Structure):
    _fields_ = [("lb", ctypes.c_double), ("ub", ctypes.c_double), ("certified", ctypes.c_int),
                ("rounds_run", ctypes.c_int), ("kept", ctypes.c_longlong * MAX_ROUNDS),
                ("pair_tests", ctypes.c_longlong * MAX_ROUNDS), ("lb_round", ctypes.c_double * MAX_ROUNDS),
                ("uv1", ctypes.c_double * 2), ("uv2", ctypes.c_double * 2), ("point1", ctypes.c_double * 3),
                ("point2", ctypes.c_double * 3), ("device_ms", ctypes.c_float)]


_lib = None


def load(path: Path | str | None = None) -> ctypes.CDLL:
    """Load libjsi_b200.so and declare its signatures (raises if absent)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} is missing: build it with `python -m jsi_cad_next_versions_b200.build` "
                           "(there is no CPU fallback)")
    L = ctypes.CDLL(str(p))
    P = ctypes.c_void_p
    I = ctypes.c_int
    L.jsi_abi_version.restype = I
    L.jsi_status_string.argtypes = [I]
    L.jsi_status_string.restype = ctypes.c_char_p
    L.jsi_last_error.argtypes = [P]
    L.jsi_last_error.restype = ctypes.c_char_p
    L.jsi_create.argtypes = [ctypes.POINTER(Config), ctypes.POINTER(P)]
    L.jsi_create.restype = I
    L.jsi_destroy.argtypes = [P]
    L.jsi_destroy.restype = I
    L.jsi_surface_upload.argtypes = [P, P, P, I, ctypes.POINTER(I)]
    L.jsi_surface_upload.restype = I
    L.jsi_host_alloc.argtypes = [P, ctypes.c_ulonglong, ctypes.POINTER(P)]
    L.jsi_host_alloc.restype = I
    L.jsi_host_free.argtypes = [P, P]
    L.jsi_host_free.restype = I
    L.jsi_surface_release.argtypes = [P, I]
    L.jsi_surface_release.restype = I
    L.jsi_resident_bytes.argtypes = [P, ctypes.POINTER(ctypes.c_ulonglong)]
    L.jsi_resident_bytes.restype = I
    L.jsi_context_stream.argtypes = [P, ctypes.POINTER(P)]
    L.jsi_context_stream.restype = I
    L.jsi_transfer_bytes.argtypes = [P, ctypes.POINTER(ctypes.c_ulonglong), ctypes.POINTER(ctypes.c_ulonglong)]
    L.jsi_transfer_bytes.restype = I
    L.jsi_launch_count.argtypes = [ctypes.POINTER(ctypes.c_ulonglong)]
    L.jsi_launch_count.restype = I
    L.jsi_kernel_timing.argtypes = [P, I]
    L.jsi_kernel_timing.restype = I
    L.jsi_kernel_time.argtypes = [P, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double),
                                  ctypes.POINTER(ctypes.c_longlong)]
    L.jsi_kernel_time.restype = I
    L.jsi_kernel_units.argtypes = [P, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double)]
    L.jsi_kernel_units.restype = I
    L.jsi_kernel_names.argtypes = [P]
    L.jsi_kernel_names.restype = ctypes.c_char_p
    L.jsi_dist_params_default.argtypes = [ctypes.POINTER(DistParams)]
    L.jsi_dist_params_default.restype = None
    L.jsi_min_distance.argtypes = [P, ctypes.POINTER(Task), ctypes.POINTER(Task), ctypes.POINTER(DistParams),
                                   ctypes.POINTER(DistResult)]
    L.jsi_min_distance.restype = I
    L.jsi_inter_params_default.argtypes = [ctypes.POINTER(InterParams)]
    L.jsi_inter_params_default.restype = None
    L.jsi_intersect.argtypes = [P, ctypes.POINTER(Task), ctypes.POINTER(Task), ctypes.POINTER(InterParams),
                                ctypes.POINTER(InterResult)]
    L.jsi_intersect.restype = I
    L.jsi_eval_grid.argtypes = [P, P, P, I, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, I, P]
    L.jsi_eval_grid.restype = I
    L.jsi_eval_grid_f64.argtypes = [P, P, P, I, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, I, P]
    L.jsi_eval_grid_f64.restype = I
    LL = ctypes.c_longlong
    L.jsi_workers.argtypes = [P, I, ctypes.c_ulonglong]
    L.jsi_workers.restype = I
    L.jsi_submit_distance.argtypes = [P, ctypes.POINTER(Task), ctypes.POINTER(Task), ctypes.POINTER(DistParams),
                                      ctypes.POINTER(ctypes.c_int), LL, ctypes.POINTER(LL)]
    L.jsi_submit_distance.restype = I
    L.jsi_submit_intersect.argtypes = [P, ctypes.POINTER(Task), ctypes.POINTER(Task), ctypes.POINTER(InterParams),
                                       ctypes.POINTER(ctypes.c_int), LL, ctypes.POINTER(LL)]
    L.jsi_submit_intersect.restype = I
    L.jsi_wait.argtypes = [P, LL, I, ctypes.POINTER(DistResult), ctypes.POINTER(InterResult)]
    L.jsi_wait.restype = I
    L.jsi_queue_depth.argtypes = [P, ctypes.POINTER(I), ctypes.POINTER(I)]
    L.jsi_queue_depth.restype = I
    L.jsi_min_distance_batch.argtypes = [P, I, ctypes.POINTER(Task), ctypes.POINTER(Task), ctypes.POINTER(DistParams),
                                         ctypes.POINTER(DistResult), ctypes.POINTER(I), ctypes.POINTER(ctypes.c_float)]
    L.jsi_min_distance_batch.restype = I
    L.jsi_submit_distance_batch.argtypes = [P, I, ctypes.POINTER(Task), ctypes.POINTER(Task), ctypes.POINTER(DistParams),
                                            ctypes.POINTER(DistResult), ctypes.POINTER(I), ctypes.POINTER(ctypes.c_longlong)]
    L.jsi_submit_distance_batch.restype = I
    L.jsi_wait_distance_batch.argtypes = [P, ctypes.c_longlong, ctypes.POINTER(ctypes.c_float)]
    L.jsi_wait_distance_batch.restype = I
    # datas: the address of an array of n float pointers
    L.jsi_surface_upload_many.argtypes = [P, I, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.jsi_surface_upload_many.restype = I
    L.jsi_surface_release_many.argtypes = [P, I, ctypes.c_void_p]
    L.jsi_surface_release_many.restype = I
    L.jsi_surface_domains.argtypes = [P, I, ctypes.c_void_p, ctypes.c_void_p]
    L.jsi_surface_domains.restype = I
    L.jsi_curve_params_default.argtypes = [ctypes.POINTER(CurveParams)]
    L.jsi_curve_params_default.restype = None
    L.jsi_intersection_curves.argtypes = [P, ctypes.POINTER(Task), ctypes.POINTER(Task), ctypes.POINTER(CurveParams),
                                          ctypes.POINTER(CurveResult)]
    L.jsi_intersection_curves.restype = I
    L.jsi_bounds_params_default.argtypes = [ctypes.POINTER(BoundsParams)]
    L.jsi_bounds_params_default.restype = None
    L.jsi_distance_bounds.argtypes = [P, ctypes.POINTER(Task), ctypes.POINTER(Task), ctypes.POINTER(BoundsParams),
                                      ctypes.POINTER(BoundsResult)]
    L.jsi_distance_bounds.restype = I
    L.jsi_batch_chunk.argtypes = [P, I]
    L.jsi_batch_chunk.restype = I
    L.jsi_batch_reruns.argtypes = [P, ctypes.POINTER(LL)]
    L.jsi_batch_reruns.restype = I
    L.jsi_batch_graphs.argtypes = [P, I, ctypes.POINTER(LL)]
    L.jsi_batch_graphs.restype = I
    L.jsi_autotune_batch.argtypes = [P, I, ctypes.POINTER(Task), ctypes.POINTER(Task), ctypes.POINTER(DistParams),
                                     ctypes.POINTER(I), ctypes.POINTER(ctypes.c_float)]
    L.jsi_autotune_batch.restype = I
    L.jsi_query_batch.argtypes = [P, I, ctypes.POINTER(I), ctypes.POINTER(Task), ctypes.POINTER(Task),
                                  ctypes.POINTER(DistParams), ctypes.POINTER(InterParams), ctypes.POINTER(DistResult),
                                  ctypes.POINTER(InterResult), ctypes.POINTER(I), ctypes.POINTER(ctypes.c_float)]
    L.jsi_query_batch.restype = I
    L.jsi_poll_distance_batch.argtypes = [P, ctypes.c_longlong, ctypes.POINTER(I)]
    L.jsi_poll_distance_batch.restype = I
    L.jsi_eval_grid_noalloc.argtypes = [P, P, I, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                        I, P]
    L.jsi_eval_grid_noalloc.restype = I
    L.jsi_surface_curvature_bounds.argtypes = [P, P, I, P, ctypes.POINTER(ctypes.c_double),
                                               ctypes.POINTER(ctypes.c_double)]
    L.jsi_surface_curvature_bounds.restype = I
    if path is None:
        _lib = L
    return L
