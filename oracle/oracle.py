"""ctypes front-end of the CPU oracle (liboracle.so) and of the reference shim (_ref/libapg_ref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg, always as the checker or the timed CPU baseline, never as the product path.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libapg_ref.so"

FAST, BALANCED, HIGH_QUALITY = 0, 1, 2


class PipelineConfig(C.Structure):
    """ctypes mirror of apg_pipeline_config_t (include/apg_sgm/pipeline_config.h)."""

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

    def copy(self) -> "PipelineConfig":
        c = PipelineConfig()
        C.pointer(c)[0] = self
        return c

    @property
    def D(self) -> int:
        return self.max_disparity - self.min_disparity


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


def telemetry_dict(rec) -> dict:
    return {k: (list(getattr(rec, k)) if k in ("delta_buckets", "route_counts", "run_length_buckets")
                else getattr(rec, k)) for k, _ in rec._fields_}


_orc = None
_ref = None


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def lib():
    global _orc
    if _orc is None:
        if not ORACLE_SO.exists():
            raise RuntimeError(f"oracle library missing: {ORACLE_SO} (run make -C oracle oracle)")
        _orc = C.CDLL(str(ORACLE_SO))
        _orc.orc_fnv1a64.restype = C.c_uint64
        _orc.orc_refine_count.restype = C.c_int
        _orc.orc_extract_supports.restype = C.c_int
        _orc.orc_rng_create.restype = C.c_void_p
        _orc.orc_rng_create.argtypes = [C.c_uint32]
        _orc.orc_rng_destroy.argtypes = [C.c_void_p]
        _orc.orc_rng_draws.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        _orc.orc_hier_range.restype = C.c_int
    return _orc


def ref_available() -> bool:
    return REF_SO.exists()


def ref_lib():
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            raise RuntimeError(f"reference library missing: {REF_SO} (run make -C oracle ref)")
        _ref = C.CDLL(str(REF_SO))
        _ref.ref_session_create.restype = C.c_void_p
        _ref.ref_session_create.argtypes = [C.POINTER(PipelineConfig), C.c_int]
        _ref.ref_session_destroy.argtypes = [C.c_void_p]
        _ref.ref_session_process.argtypes = [C.c_void_p] + [C.c_void_p] * 2 + [C.c_int] * 4 + [C.c_void_p] * 6
        _ref.ref_max_threads.restype = C.c_int
    return _ref


def config(mode: int, max_disparity: int = 128, min_disparity: int = 0, **kw) -> PipelineConfig:
    """PipelineConfig::from_mode(mode, max_disparity) (src/config.cpp:5-45) plus overrides."""
    c = PipelineConfig()
    lib().orc_config_from_mode(C.c_int(mode), C.c_int(max_disparity), C.byref(c))
    c.min_disparity = min_disparity
    for k, v in kw.items():
        if not hasattr(c, k):
            raise AttributeError(k)
        setattr(c, k, v)
    return c


def config_from_record(raw: bytes) -> PipelineConfig:
    """A configuration saved as the raw bytes of apg_pipeline_config_t.  Records shorter than the
    current struct (saved before the hierarchical fields were appended) keep the from_mode
    defaults of the fields after them."""
    c = config(BALANCED, 128)
    C.memmove(C.addressof(c), raw, min(len(raw), C.sizeof(c)))
    return c


def fnv1a64(a: np.ndarray) -> int:
    a = np.ascontiguousarray(a)
    return int(lib().orc_fnv1a64(_p(a), C.c_uint64(a.nbytes)))


def _as_u8(img):
    img = np.asarray(img)
    assert img.dtype == np.uint8
    return img


def _view(img):
    """(contiguous-rows array, w, h, stride, channels) of an HxW or HxWxC uint8 array."""
    img = _as_u8(img)
    h, w = img.shape[:2]
    ch = 1 if img.ndim == 2 else img.shape[2]
    if not (img.strides[-1] == 1 and (img.ndim == 2 or img.strides[1] == ch)):
        img = np.ascontiguousarray(img)
    stride = img.strides[0]
    return img, w, h, stride, ch


class _OrcStages(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in ("disp_wta", "best", "second", "disp_right", "disp_refined",
                                          "disp_lr", "disp_fill", "cost_raw", "cost_agg", "sgm_sum",
                                          "range_min", "range_max", "d_prior")] + [("support_count", C.c_int)]


def pipeline(cfg: PipelineConfig, left, right, stages: bool = False) -> dict:
    """Oracle whole-pipeline run (Dense semantics).  Returns final outputs and, optionally,
    every intermediate of orc_stages_t."""
    L, w, h, stride, ch = _view(left)
    R, _, _, _, _ = _view(right)
    D = cfg.D
    out = {
        "disparity": np.empty((h, w), np.float32), "confidence": np.empty((h, w), np.float32),
        "invalid_reason": np.empty((h, w), np.uint8), "reliable_mask": np.empty((h, w), np.uint8),
    }
    st = None
    if stages:
        out.update({
            "disp_wta": np.empty((h, w), np.float32), "best": np.empty((h, w), np.float32),
            "second": np.empty((h, w), np.float32), "disp_right": np.empty((h, w), np.float32),
            "disp_refined": np.empty((h, w), np.float32), "disp_lr": np.empty((h, w), np.float32),
            "disp_fill": np.empty((h, w), np.float32),
            "cost_raw": np.empty((h, w, D), np.uint16), "cost_agg": np.empty((h, w, D), np.uint16),
            "sgm_sum": np.empty((h, w, D), np.uint32),
            "range_min": np.empty((h, w), np.int16), "range_max": np.empty((h, w), np.int16),
            "d_prior": np.empty((h, w), np.float32),
        })
        st = _OrcStages()
        for k, _ in _OrcStages._fields_[:-1]:
            setattr(st, k, out[k].ctypes.data)
    rc = lib().orc_pipeline(C.byref(cfg), _p(L), _p(R), w, h, stride, ch,
                            _p(out["disparity"]), _p(out["confidence"]), _p(out["invalid_reason"]),
                            _p(out["reliable_mask"]), C.byref(st) if stages else None)
    if stages:
        out["support_count"] = st.support_count
    out["status"] = rc
    return out


def hier_range(cfg: PipelineConfig, left, right) -> dict:
    """Oracle hierarchical search range (orc_hier_range): range planes, d_prior, the coarse
    pass's disparity and confidence, and the telemetry numerators."""
    a = aux(left, right)
    h, w = a["left"]["gray"].shape
    wc, hc = w // 2, h // 2
    out = {"range_min": np.empty((h, w), np.int16), "range_max": np.empty((h, w), np.int16),
           "d_prior": np.empty((h, w), np.float32), "coarse_disparity": np.full((max(hc, 1), max(wc, 1)), -1, np.float32),
           "coarse_confidence": np.zeros((max(hc, 1), max(wc, 1)), np.float32)}
    cnt = np.zeros(4, np.int64)
    ran = lib().orc_hier_range(C.byref(cfg), w, h, _p(a["left"]["gray"]), _p(a["right"]["gray"]),
                               _p(out["range_min"]), _p(out["range_max"]), _p(out["d_prior"]), _p(cnt),
                               _p(out["coarse_disparity"]), _p(out["coarse_confidence"]))
    out["ran"] = int(ran)
    out["coarse_valid"], out["fallback"], out["full_range"], out["width_sum"] = (int(v) for v in cnt)
    n = w * h
    out["telemetry"] = {"avg_states_per_pixel": out["width_sum"] / n if n else 0.0,
                        "coarse_valid_ratio": float(np.float32(out["coarse_valid"] / (wc * hc))) if ran else 0.0,
                        "fallback_pixel_ratio": float(np.float32(out["fallback"] / n)),
                        "full_range_pixel_ratio": float(np.float32(out["full_range"] / n))}
    return out


def hier_coarse_config(cfg: PipelineConfig) -> PipelineConfig:
    c = PipelineConfig()
    lib().orc_hier_coarse_config(C.byref(cfg), C.byref(c))
    return c


def aux(left, right):
    """gray, gx, gy, census(sym) of both images (oracle)."""
    res = {}
    for side, img in (("left", left), ("right", right)):
        I, w, h, stride, ch = _view(img)
        g = np.empty((h, w), np.uint8); gx = np.empty_like(g); gy = np.empty_like(g)
        lib().orc_gray_grad(_p(I), w, h, stride, ch, _p(g), _p(gx), _p(gy))
        cs = np.empty((h, w), np.uint32)
        lib().orc_census_sym(_p(g), w, h, _p(cs))
        c64 = np.empty((h, w), np.uint64)
        lib().orc_census64(_p(g), w, h, _p(c64))
        res[side] = {"gray": g, "gx": gx, "gy": gy, "census": cs, "census64": c64}
    return res


def sgm_path(cfg: PipelineConfig, gray, vol, acc, dx, dy):
    h, w, D = vol.shape
    lib().orc_sgm_path(C.byref(cfg), _p(gray), _p(vol), _p(acc), w, h, D, dx, dy)


def wta(cfg: PipelineConfig, acc, rmin, rmax):
    h, w, _ = acc.shape
    disp = np.empty((h, w), np.float32); best = np.empty_like(disp); second = np.empty_like(disp)
    lib().orc_wta(C.byref(cfg), _p(acc), _p(rmin), _p(rmax), w, h, _p(disp), _p(best), _p(second))
    return disp, best, second


def wta_right(cfg: PipelineConfig, raw):
    """Right-image disparity from the raw cost volume, (h, w, D) u16 (orc_wta_right, the restatement
    of wta_right_from_left_volume, src/pipeline.cpp:24-85)."""
    raw = np.ascontiguousarray(raw, np.uint16)
    h, w, _ = raw.shape
    out = np.empty((h, w), np.float32)
    lib().orc_wta_right(C.byref(cfg), _p(raw), w, h, _p(out))
    return out


def rng_draws(seed: int, plan):
    """Concatenated draws of std::uniform_int_distribution(-r, r) over one mt19937(seed) for a
    list of (radius, count) pairs."""
    L = lib()
    h = L.orc_rng_create(C.c_uint32(seed))
    try:
        outs = []
        for r, n in plan:
            a = np.empty(max(n, 1), np.int32)
            L.orc_rng_draws(h, int(r), int(n), _p(a))
            outs.append(a[:n])
        return outs
    finally:
        L.orc_rng_destroy(h)


# ----------------------------------------------------------------------------------------------
# Reference (oracle/_ref) front-end
# ----------------------------------------------------------------------------------------------

_DUMP_FIELDS = [
    ("left_gray", np.uint8, 2), ("left_gx", np.uint8, 2), ("left_gy", np.uint8, 2),
    ("right_gray", np.uint8, 2), ("right_gx", np.uint8, 2), ("right_gy", np.uint8, 2),
    ("census_left", np.uint32, 2), ("census_right", np.uint32, 2),
    ("census_left64", np.uint64, 2), ("census_right64", np.uint64, 2),
    ("range_min", np.int16, 2), ("range_max", np.int16, 2),
    ("cost_raw", np.uint16, 3), ("cost_agg", np.uint16, 3), ("sgm_sum", np.uint32, 3),
    ("disp_wta", np.float32, 2), ("best", np.float32, 2), ("second", np.float32, 2),
    ("disp_right", np.float32, 2),
    ("conf_confidence", np.float32, 2), ("conf_reliable", np.uint8, 2), ("conf_reason", np.uint8, 2),
    ("d_prior", np.float32, 2), ("disp_refined", np.float32, 2),
    ("disp_lr", np.float32, 2), ("reason_lr", np.uint8, 2), ("disp_fill", np.float32, 2),
    ("disparity", np.float32, 2), ("confidence", np.float32, 2),
    ("invalid_reason", np.uint8, 2), ("reliable_mask", np.uint8, 2),
]
_DUMP_TAIL = [("prior_conf", np.float32, 2), ("prior_spread", np.float32, 2),
              ("prior_dmin", np.float32, 2), ("prior_dmax", np.float32, 2)]


class _RefDump(C.Structure):
    _fields_ = [(n, C.c_void_p) for n, _, _ in _DUMP_FIELDS] + [("support_count", C.c_int)] + \
               [(n, C.c_void_p) for n, _, _ in _DUMP_TAIL]


def ref_dump(cfg: PipelineConfig, left, right) -> dict:
    """Every stage output of the reference Dense pipeline on (left, right)."""
    L, w, h, stride, ch = _view(left)
    R, _, _, _, _ = _view(right)
    D = cfg.D
    out, d = {}, _RefDump()
    sym = cfg.census_type == 1
    for name, dt, nd in _DUMP_FIELDS + _DUMP_TAIL:
        if name.endswith("64") and sym or (name in ("census_left", "census_right") and not sym):
            continue
        a = np.zeros((h, w, D) if nd == 3 else (h, w), dt)
        out[name] = a
        setattr(d, name, a.ctypes.data)
    rc = ref_lib().ref_dump(C.byref(cfg), _p(L), _p(R), w, h, stride, ch, C.byref(d))
    out["status"] = rc
    out["support_count"] = d.support_count
    return out


def ref_hier_dump(cfg: PipelineConfig, left, right) -> dict:
    """The reference's hierarchical search range (range planes, d_prior, telemetry) and the final
    maps of its full pipeline with the same configuration (ref_hier_dump in ref_shim.cpp)."""
    L, w, h, stride, ch = _view(left)
    R, _, _, _, _ = _view(right)
    out = {"range_min": np.zeros((h, w), np.int16), "range_max": np.zeros((h, w), np.int16),
           "d_prior": np.zeros((h, w), np.float32),
           "disparity": np.zeros((h, w), np.float32), "confidence": np.zeros((h, w), np.float32),
           "invalid_reason": np.zeros((h, w), np.uint8), "reliable_mask": np.zeros((h, w), np.uint8)}
    t = np.zeros(5, np.float64)
    rc = ref_lib().ref_hier_dump(C.byref(cfg), _p(L), _p(R), w, h, stride, ch, _p(out["range_min"]),
                                 _p(out["range_max"]), _p(out["d_prior"]), _p(t), _p(out["disparity"]),
                                 _p(out["confidence"]), _p(out["invalid_reason"]), _p(out["reliable_mask"]))
    out["status"] = rc
    out["ran"] = int(t[4])
    out["telemetry"] = dict(zip(["avg_states_per_pixel", "coarse_valid_ratio", "fallback_pixel_ratio",
                                 "full_range_pixel_ratio"], t[:4].tolist()))
    return out


def _metric_args(est, gt, range_, before, after, vis, left):
    est = np.ascontiguousarray(est, np.float32)
    gt = np.ascontiguousarray(gt, np.float32)
    h, w = gt.shape
    rmin = rmax = None
    if range_ is not None:
        rmin, rmax = (np.ascontiguousarray(a, np.int16) for a in range_)
    if before is not None:
        before, after = np.ascontiguousarray(before, np.float32), np.ascontiguousarray(after, np.float32)
    if vis is not None:
        vis = np.ascontiguousarray(vis, np.uint8)
    lstride = lch = 0
    if left is not None:
        left = np.ascontiguousarray(left, np.uint8)
        lch = 1 if left.ndim == 2 else left.shape[2]
        lstride = w * lch
    keep = (est, gt, rmin, rmax, before, after, vis, left)
    return keep, w, h, lstride, lch


def _thr(thresholds):
    if thresholds is None:
        return None
    t = QualityThresholdsRec()
    t.boundary_disparity_gradient, t.low_texture_gradient, t.max_valid_gt = thresholds
    return C.byref(t)


def evaluate_stereo(est, gt, range_=None, before=None, after=None, vis=None, max_valid_gt=1e5, left=None,
                    thresholds=None, reference=False) -> StereoMetricsRec:
    """evaluate_stereo (src/metrics.cpp:119-502, no supports): the oracle's restatement, or with
    reference=True the reference build's own function.  thresholds: (boundary, low_texture, max_gt)."""
    keep, w, h, lstride, lch = _metric_args(est, gt, range_, before, after, vis, left)
    out = StereoMetricsRec()
    f = ref_lib().ref_evaluate_stereo if reference else lib().orc_evaluate_stereo
    f(*[_p(a) for a in keep[:2]], C.c_int(w), C.c_int(h), *[_p(a) for a in keep[2:7]], C.c_float(max_valid_gt),
      _p(keep[7]), C.c_int(lstride), C.c_int(lch), _thr(thresholds), C.byref(out))
    return out


def ref_load_image(path):
    """The reference's load_image: (status, array or None); status 1 ok, 0 failed, -1 threw."""
    w, h, c = C.c_int(), C.c_int(), C.c_int()
    rc = ref_lib().ref_load_image(str(path).encode(), None, C.c_size_t(0), C.byref(w), C.byref(h), C.byref(c))
    if rc != 1:
        return rc, None
    a = np.empty((h.value, w.value, c.value) if c.value > 1 else (h.value, w.value), np.uint8)
    ref_lib().ref_load_image(str(path).encode(), _p(a), C.c_size_t(a.nbytes), C.byref(w), C.byref(h), C.byref(c))
    return 1, a


def ref_load_pfm(path):
    w, h = C.c_int(), C.c_int()
    rc = ref_lib().ref_load_pfm(str(path).encode(), None, C.c_size_t(0), C.byref(w), C.byref(h))
    if rc != 1:
        return rc, None
    a = np.empty((h.value, w.value), np.float32)
    ref_lib().ref_load_pfm(str(path).encode(), _p(a), C.c_size_t(a.size), C.byref(w), C.byref(h))
    return 1, a


def ref_save(kind: str, path, arr, dmax: float = 0.0) -> int:
    """The reference's save_pgm / save_pgm16 / save_disparity_preview / save_pfm."""
    a = np.ascontiguousarray(arr)
    h, w = a.shape[:2]
    f = getattr(ref_lib(), "ref_save_" + kind)
    args = [str(path).encode(), _p(a), C.c_int(w), C.c_int(h)]
    if kind == "disparity_preview":
        args.append(C.c_float(dmax))
    return int(f(*args))


def evaluate_supports(x, y, d, gt, vis=None, max_valid_gt=1e5, cell_size=16, reference=False) -> SupportMetricsRec:
    """evaluate_supports (src/metrics.cpp:8-124): the oracle's, or with reference=True the reference's."""
    gt = np.ascontiguousarray(gt, np.float32)
    h, w = gt.shape
    out = SupportMetricsRec()
    if vis is not None:
        vis = np.ascontiguousarray(vis, np.uint8)
    if reference:
        xs, ys, ds = (np.ascontiguousarray(a, t) for a, t in ((x, np.int32), (y, np.int32), (d, np.float32)))
        ref_lib().ref_evaluate_supports(_p(xs), _p(ys), _p(ds), C.c_int(len(xs)), _p(gt), C.c_int(w), C.c_int(h),
                                        _p(vis), C.c_float(max_valid_gt), C.c_int(cell_size), C.byref(out))
    else:
        n = len(x)
        sp = np.zeros(n, dtype=[("x", "<i4"), ("y", "<i4"), ("d", "<f4"), ("c", "<f4")])
        sp["x"], sp["y"], sp["d"] = x, y, d
        lib().orc_evaluate_supports(_p(sp), C.c_int(n), _p(gt), C.c_int(w), C.c_int(h), _p(vis),
                                    C.c_float(max_valid_gt), C.c_int(cell_size), C.byref(out))
    return out


def supports(cfg: PipelineConfig, left, right):
    """The oracle prior's selected supports of a pair, in order: (x, y, disparity, confidence) arrays."""
    a = aux(left, right)
    h, w = a["left"]["gray"].shape
    cap = max(1, cfg.prior_max_supports)
    sp = np.zeros(cap, dtype=[("x", "<i4"), ("y", "<i4"), ("d", "<f4"), ("c", "<f4")])
    sym = cfg.census_type == 1
    n = lib().orc_extract_supports(C.byref(cfg), w, h, _p(a["left"]["gx"]), _p(a["left"]["gy"]),
                                   _p(a["left"]["census"]) if sym else None, _p(a["right"]["census"]) if sym else None,
                                   None if sym else _p(a["left"]["census64"]),
                                   None if sym else _p(a["right"]["census64"]), _p(sp), cap)
    sp = sp[:n]
    return sp["x"].copy(), sp["y"].copy(), sp["d"].copy(), sp["c"].copy()


def set_experimental(sp_method: int = 0, sp_param: float = 0.0, ip_method: int = 0, ip_gap: int = 32,
                     reference: bool = False, sp_telemetry: bool = False, ip_telemetry: bool = False):
    """The experimental scopes (sub-pixel method/param, inpaint method/gap, telemetry on/off: on
    clears the totals) of the oracle, or with reference=True the reference's own scopes on the
    calling thread."""
    if reference:
        ref_lib().ref_set_experimental_tel(C.c_int(sp_method), C.c_float(sp_param), C.c_int(int(sp_telemetry)),
                                           C.c_int(ip_method), C.c_int(ip_gap), C.c_int(int(ip_telemetry)))
    else:
        lib().orc_set_experimental(C.c_int(sp_method), C.c_float(sp_param), C.c_int(ip_method), C.c_int(ip_gap))
        lib().orc_set_telemetry(C.c_int(int(sp_telemetry)), C.c_int(int(ip_telemetry)))


def get_telemetry(reference: bool = False):
    """(sub-pixel, inpaint) telemetry totals as dicts: the oracle's or the reference's."""
    sp, ip = SubpixelTelemetryRec(), InpaintTelemetryRec()
    (ref_lib().ref_get_telemetry if reference else lib().orc_get_telemetry)(C.byref(sp), C.byref(ip))
    return telemetry_dict(sp), telemetry_dict(ip)


class RefSession:
    """The reference's public StereoSession (BoundedReuse) for timing its CPU path."""

    def __init__(self, cfg: PipelineConfig, bounded_reuse: bool = True):
        self._h = ref_lib().ref_session_create(C.byref(cfg), 1 if bounded_reuse else 0)

    def process(self, left, right, want_stages=False):
        L, w, h, stride, ch = _view(left)
        R, _, _, _, _ = _view(right)
        out = {"disparity": np.empty((h, w), np.float32), "confidence": np.empty((h, w), np.float32),
               "invalid_reason": np.empty((h, w), np.uint8), "reliable_mask": np.empty((h, w), np.uint8)}
        st = np.zeros(11, np.float64)
        fs = np.zeros(13, np.float64)
        rc = ref_lib().ref_session_process(self._h, _p(L), _p(R), w, h, stride, ch,
                                           _p(out["disparity"]), _p(out["confidence"]),
                                           _p(out["invalid_reason"]), _p(out["reliable_mask"]), _p(st), _p(fs))
        out["status"] = rc
        out["stage_ms"] = dict(zip(["aux", "prior", "cost", "cross", "right_wta", "sgm", "wta",
                                    "confidence", "refine", "post", "total"], st.tolist()))
        out["stats"] = dict(zip(["valid_pixels", "reliable_pixels", "unreliable_pixels", "refine_changed_pixels",
                                 "lr_fail_pixels", "prior_support_count", "mean_search_width",
                                 "mean_geometry_width", "valid_disparity_ratio", "reliable_ratio",
                                 "unreliable_ratio", "refine_changed_ratio", "lr_fail_ratio"], fs.tolist()))
        return out

    def close(self):
        if self._h:
            ref_lib().ref_session_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ref_threads() -> int:
    return int(ref_lib().ref_max_threads())
