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


_REGION_FIELDS = ["total_pixels", "valid_est_pixels", "valid_ratio", "epe", "bad_0_5", "bad_1_0", "bad_2_0",
                  "bad_3_0", "d1"]


class RegionMetricsRec(C.Structure):
    """apg_region_metrics_t (include/apg_sgm/metrics.h): RegionMetrics."""
    _fields_ = [(k, C.c_int if k in ("total_pixels", "valid_est_pixels") else C.c_float) for k in _REGION_FIELDS]


class QualityThresholdsRec(C.Structure):
    """apg_quality_thresholds_t (include/apg_sgm/metrics.h): QualityThresholds."""
    _fields_ = [("boundary_disparity_gradient", C.c_float), ("low_texture_gradient", C.c_float),
                ("max_valid_gt", C.c_float)]


_I, _F, _U = C.c_int, C.c_float, C.c_ulonglong
_STEREO_FIELDS = (
    [("total_pixels", _I), ("evaluated_pixels", _I), ("valid_pixels", _I), ("valid_ratio", _F), ("epe", _F),
     ("bad_0_5", _F), ("bad_1_0", _F), ("bad_2_0", _F), ("bad_3_0", _F), ("kitti_d1_all", _F), ("kitti_d1_noc", _F),
     ("edge_pixels", _I), ("edge_epe", _F), ("nonedge_pixels", _I), ("nonedge_epe", _F), ("lr_fail_ratio", _F),
     ("has_range", _I), ("range_recall_all", _F), ("range_recall_matchable", _F), ("range_recall_visible", _F),
     ("range_visible_eval_pixels", _U), ("range_visible_in_pixels", _U), ("range_matchable_eval_pixels", _U),
     ("range_matchable_in_pixels", _U), ("prior_miss_visible_count", _I), ("prior_miss_edge", _I),
     ("prior_miss_nonedge", _I), ("prior_miss_edge_ratio", _F), ("prior_miss_nonedge_ratio", _F)]
    + [(r, RegionMetricsRec) for r in ("reg_all", "reg_noc", "reg_occ", "reg_boundary", "reg_non_boundary",
                                       "reg_low_texture", "reg_high_texture")]
    + [("has_refine_stats", _I), ("refine_eval_pixels", _I), ("refine_epe_delta", _F), ("post_epe_delta", _F),
       ("total_epe_delta", _F), ("refine_improved_ratio", _F), ("refine_worsened_ratio", _F),
       ("refine_unchanged_ratio", _F), ("refine_changed_ratio", _F)])


class StereoMetricsRec(C.Structure):
    """apg_stereo_metrics_t (include/apg_sgm/metrics.h): StereoMetrics without the support block."""
    _fields_ = _STEREO_FIELDS

    def to_dict(self) -> dict:
        d = {}
        for k, t in self._fields_:
            v = getattr(self, k)
            d[k] = {r: getattr(v, r) for r in _REGION_FIELDS} if t is RegionMetricsRec else v
        return d


_SUPPORT_INT = ["total", "gt_valid", "visible", "correct_05", "correct_1", "correct_2", "visible_correct_05",
                "visible_correct_1", "visible_correct_2", "visible_gt_cells", "correct_visible_cells"]
_SUPPORT_FLOAT = ["precision_05", "precision_1", "precision_2", "precision_all_05", "precision_all_1",
                  "precision_all_2", "precision_vis_05", "precision_vis_1", "precision_vis_2", "mean_abs_error",
                  "mae_all", "mae_visible", "grid_recall_1", "grid_coverage", "support_grid_recall_vis_1"]


class SupportMetricsRec(C.Structure):
    """apg_support_metrics_t (include/apg_sgm/metrics.h): SupportMetrics."""
    _fields_ = [(k, C.c_int) for k in _SUPPORT_INT] + [(k, C.c_float) for k in _SUPPORT_FLOAT]

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


class SubpixelTelemetryRec(C.Structure):
    """apg_subpixel_telemetry_t (include/apg_sgm/telemetry.h)."""
    _fields_ = [("candidate_pixels", C.c_ulonglong), ("applied_pixels", C.c_ulonglong),
                ("degenerate_count", C.c_ulonglong), ("clamped_count", C.c_ulonglong),
                ("negative_curvature_count", C.c_ulonglong), ("sum_abs_delta", C.c_double),
                ("delta_buckets", C.c_ulonglong * 50)]


class InpaintTelemetryRec(C.Structure):
    """apg_inpaint_telemetry_t (include/apg_sgm/telemetry.h)."""
    _fields_ = [("total_invalid_pixels", C.c_ulonglong), ("classified_occ_pixels", C.c_ulonglong),
                ("classified_mismatch_pixels", C.c_ulonglong), ("hit_max_gap_pixels", C.c_ulonglong),
                ("reclassified_shadow_pixels", C.c_ulonglong), ("route_counts", C.c_ulonglong * 11),
                ("invalid_runs_count", C.c_ulonglong), ("invalid_runs_truncated", C.c_ulonglong),
                ("run_length_buckets", C.c_ulonglong * 10)]


class LoadedPair(C.Structure):
    """apgcu_loaded_pair_t (include/apg_sgm_cuda.h): one pair read by the loader."""
    _fields_ = [("status", C.c_int), ("width", C.c_int), ("height", C.c_int), ("channels", C.c_int),
                ("left", C.c_void_p), ("right", C.c_void_p)]


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
    "apgcu_session_set_tuning": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int]),
    "apgcu_session_estimate_bytes": (C.c_size_t, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "apgcu_session_get_frame_counts": (C.c_int, [C.c_void_p, C.POINTER(C.c_ulonglong)]),
    "apgcu_session_hier_telemetry": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "apgcu_engine_hier_telemetry": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "apgcu_kernel_launch_count": (C.c_ulonglong, []),
    "apgcu_evaluate_supports": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                          C.c_void_p, C.c_float, C.c_int, C.c_int, C.c_void_p,
                                          C.POINTER(SupportMetricsRec)]),
    "apgcu_engine_supports": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "apgcu_set_experimental": (C.c_int, [C.c_int, C.c_float, C.c_int, C.c_int]),
    "apgcu_set_experimental_telemetry": (C.c_int, [C.c_int, C.c_int]),
    "apgcu_get_experimental_telemetry": (None, [C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "apgcu_get_telemetry": (None, [C.c_void_p, C.c_void_p]),
    "apgcu_reset_telemetry": (None, [C.c_int, C.c_int]),
    "apgcu_get_experimental": (None, [C.POINTER(C.c_int), C.POINTER(C.c_float), C.POINTER(C.c_int),
                                      C.POINTER(C.c_int)]),
    "apgcu_image_info": (C.c_int, [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "apgcu_load_image": (C.c_int, [C.c_char_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                   C.POINTER(C.c_int)]),
    "apgcu_save_pgm": (C.c_int, [C.c_char_p, C.c_void_p, C.c_int, C.c_int]),
    "apgcu_save_pgm16": (C.c_int, [C.c_char_p, C.c_void_p, C.c_int, C.c_int]),
    "apgcu_save_disparity_preview": (C.c_int, [C.c_char_p, C.c_void_p, C.c_int, C.c_int, C.c_float]),
    "apgcu_pfm_info": (C.c_int, [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "apgcu_load_pfm": (C.c_int, [C.c_char_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "apgcu_save_pfm": (C.c_int, [C.c_char_p, C.c_void_p, C.c_int, C.c_int]),
    "apgcu_loader_create": (C.c_void_p, [C.c_int]),
    "apgcu_loader_destroy": (None, [C.c_void_p]),
    "apgcu_loader_submit": (C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.POINTER(C.c_ulonglong)]),
    "apgcu_loader_wait": (C.c_int, [C.c_void_p, C.c_ulonglong, C.POINTER(LoadedPair)]),
    "apgcu_loader_release": (C.c_int, [C.c_void_p, C.c_ulonglong]),
    "apgcu_loader_pinned_bytes": (C.c_size_t, [C.c_void_p]),
    "apgcu_metrics_last_kernel_ms": (C.c_float, []),
    "apgcu_evaluate_stereo": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_float, C.c_void_p, C.c_int, C.c_int,
                                        C.POINTER(QualityThresholdsRec), C.c_int, C.c_void_p,
                                        C.POINTER(StereoMetricsRec)]),
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
