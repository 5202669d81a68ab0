"""ctypes binding of libapg_sgm_b200.so (built in-tree by apg_sgm_b200/build.py).

The library is the only compute path: if it is missing or fails to load, every entry point
raises; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libapg_sgm_b200.so"


class PipelineConfig(C.Structure):
    """ctypes mirror of apg_pipeline_config_t (include/apg_sgm/pipeline_config.h), the plain-C
    form of the reference's PipelineConfig (include/apg_sgm/config.hpp:7-112)."""

    _fields_ = [
        ("mode", C.c_int), ("min_disparity", C.c_int), ("max_disparity", C.c_int),
        ("num_threads", C.c_int), ("volume_backend", C.c_int),
        ("census_type", C.c_int),
        ("lambda_census", C.c_float), ("lambda_ad", C.c_float), ("lambda_grad", C.c_float),
        ("eta_ad", C.c_float), ("mu_grad", C.c_float),
        ("use_ad", C.c_int), ("use_grad", C.c_int), ("cost_max", C.c_int),
        ("agg_enable", C.c_int), ("max_arm_length", C.c_int), ("color_threshold", C.c_int),
        ("agg_iterations", C.c_int),
        ("paths", C.c_int), ("P1", C.c_int), ("P2_base", C.c_int), ("adaptive_penalties", C.c_int),
        ("grad_t1", C.c_int), ("grad_t2", C.c_int), ("p2_alpha", C.c_float), ("piecewise_p2", C.c_int),
        ("prior_enable", C.c_int), ("prior_uniqueness_ratio", C.c_float),
        ("prior_texture_threshold", C.c_int), ("prior_lr_max_diff", C.c_int),
        ("prior_search_radius", C.c_int), ("prior_min_supports", C.c_int),
        ("prior_max_supports", C.c_int),
        ("conf_uniqueness_ratio", C.c_float), ("conf_lr_max_diff", C.c_int),
        ("conf_min_texture", C.c_float), ("conf_reliable_threshold", C.c_float),
        ("refine_enable", C.c_int), ("refine_iterations", C.c_int), ("refine_random_radius", C.c_int),
        ("subpixel", C.c_int), ("lr_check", C.c_int), ("post_lr_max_diff", C.c_int),
        ("median_radius", C.c_int), ("max_fill_gap", C.c_int),
        ("hier_enable", C.c_int), ("hier_radius", C.c_int), ("hier_scale", C.c_int), ("hier_fallback", C.c_int),
        ("hier_coarse_cross_agg", C.c_int), ("hier_coarse_fill_holes", C.c_int),
        ("hier_adaptive_radius", C.c_int), ("hier_confidence_threshold", C.c_float),
        ("hier_expanded_radius", C.c_int),
    ]

    @property
    def D(self) -> int:
        return self.max_disparity - self.min_disparity

    def to_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class ImageView(C.Structure):
    """apg_image_view_t (include/apg_sgm/c_api.h)."""
    _fields_ = [("data", C.c_void_p), ("width", C.c_int), ("height", C.c_int),
                ("stride", C.c_int), ("channels", C.c_int)]


class SessionOptions(C.Structure):
    """apg_session_options_t (include/apg_sgm/c_api.h)."""
    _fields_ = [("struct_size", C.c_uint32), ("quality_mode", C.c_int), ("memory_policy", C.c_int),
                ("max_retained_bytes", C.c_size_t), ("num_threads", C.c_int), ("backend", C.c_int),
                ("min_disparity", C.c_int), ("max_disparity", C.c_int)]


class Pair(C.Structure):
    """apgcu_pair_t (include/apg_sgm_cuda.h): one pair of a batch."""
    _fields_ = [("left", C.c_void_p), ("right", C.c_void_p), ("width", C.c_int), ("height", C.c_int),
                ("stride", C.c_int), ("channels", C.c_int), ("max_disparity", C.c_int),
                ("disparity", C.c_void_p), ("confidence", C.c_void_p), ("invalid_reason", C.c_void_p),
                ("reliable_mask", C.c_void_p)]


class Request(C.Structure):
    """apgcu_request_t (include/apg_sgm_cuda.h): one request to the server."""
    _fields_ = [("mode", C.c_int), ("min_disparity", C.c_int), ("max_disparity", C.c_int),
                ("left", C.c_void_p), ("right", C.c_void_p), ("width", C.c_int), ("height", C.c_int),
                ("stride", C.c_int), ("channels", C.c_int), ("disparity", C.c_void_p), ("confidence", C.c_void_p),
                ("invalid_reason", C.c_void_p), ("reliable_mask", C.c_void_p)]


_lib = None

_SIGS = {
    # reference C API
    "apg_session_create": (C.c_void_p, [C.c_int, C.c_int]),
    "apg_session_create_ex": (C.c_void_p, [C.POINTER(SessionOptions)]),
    "apg_session_destroy": (None, [C.c_void_p]),
    "apg_session_reset": (None, [C.c_void_p]),
    "apg_result_create": (C.c_void_p, []),
    "apg_result_destroy": (None, [C.c_void_p]),
    "apg_session_process": (C.c_int, [C.c_void_p, C.POINTER(ImageView), C.POINTER(ImageView), C.c_void_p]),
    "apg_result_get_disparity": (C.c_void_p, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "apg_result_get_confidence": (C.c_void_p, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "apg_result_get_invalid_reason": (C.c_void_p, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "apg_result_get_reliable_mask": (C.c_void_p, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "apg_session_get_last_error": (C.c_char_p, [C.c_void_p]),
    "apg_session_get_allocated_bytes": (C.c_size_t, [C.c_void_p]),
    "apg_session_get_frame_count": (C.c_size_t, [C.c_void_p]),
    "apg_session_get_total_time_ms": (C.c_double, [C.c_void_p]),
    "apg_status_string": (C.c_char_p, [C.c_int]),
    "apg_version_string": (C.c_char_p, []),
    # extensions
    "apgcu_engine_create": (C.c_void_p, [C.POINTER(PipelineConfig), C.c_int, C.c_void_p]),
    "apgcu_engine_destroy": (None, [C.c_void_p]),
    "apgcu_engine_last_error": (C.c_char_p, [C.c_void_p]),
    "apgcu_engine_set_debug": (C.c_int, [C.c_void_p, C.c_int]),
    "apgcu_engine_set_tuning": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int]),
    "apgcu_engine_process": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "apgcu_engine_process_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                              C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "apgcu_engine_sync": (C.c_int, [C.c_void_p]),
    "apgcu_engine_dump": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]),
    "apgcu_engine_stage_times": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "apgcu_engine_allocated_bytes": (C.c_size_t, [C.c_void_p]),
    "apgcu_workspace_bytes": (C.c_size_t, [C.POINTER(PipelineConfig), C.c_int, C.c_int]),
    "apgcu_engine_release": (None, [C.c_void_p]),
    "apgcu_engine_stream": (C.c_void_p, [C.c_void_p]),
    "apgcu_config_from_mode": (None, [C.c_int, C.c_int, C.POINTER(PipelineConfig)]),
    "apgcu_session_create_config": (C.c_void_p, [C.POINTER(PipelineConfig), C.c_int, C.c_size_t]),
    "apgcu_session_get_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_size_t)]),
    "apgcu_session_estimate_bytes": (C.c_size_t, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "apgcu_session_get_frame_counts": (C.c_int, [C.c_void_p, C.POINTER(C.c_ulonglong)]),
    "apgcu_session_hier_telemetry": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "apgcu_engine_hier_telemetry": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "apgcu_kernel_launch_count": (C.c_ulonglong, []),
    "apgcu_engine_launch_profile": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_char_p), C.POINTER(C.c_float)]),
    "apgcu_batch_create": (C.c_void_p, [C.POINTER(PipelineConfig), C.c_int]),
    "apgcu_batch_destroy": (None, [C.c_void_p]),
    "apgcu_batch_last_error": (C.c_char_p, [C.c_void_p]),
    "apgcu_batch_process": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(Pair), C.c_int]),
    "apgcu_batch_set_option": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int]),
    "apgcu_batch_allocated_bytes": (C.c_size_t, [C.c_void_p]),
    "apgcu_batch_last_time_ms": (C.c_float, [C.c_void_p]),
    "apgcu_batch_release": (None, [C.c_void_p]),
    "apgcu_server_create": (C.c_void_p, [C.c_int, C.c_size_t, C.c_int]),
    "apgcu_server_destroy": (None, [C.c_void_p]),
    "apgcu_server_submit": (C.c_int, [C.c_void_p, C.POINTER(Request), C.POINTER(C.c_ulonglong)]),
    "apgcu_server_wait": (C.c_int, [C.c_void_p, C.c_ulonglong, C.POINTER(C.c_double)]),
    "apgcu_server_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_ulonglong), C.POINTER(C.c_size_t)]),
    "apgcu_server_budget": (C.c_size_t, [C.c_void_p]),
    "apgcu_server_reserve": (C.c_int, [C.c_void_p, C.POINTER(Request), C.c_int]),
    "apgcu_server_last_error": (C.c_char_p, [C.c_void_p]),
    "apgcu_right_wta_noalloc": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                          C.c_void_p, C.c_void_p]),
}


def lib():
    """Load the CUDA library (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing; build it with `python -m apg_sgm_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def declared_symbols():
    return list(_SIGS)
