"""apg_sgm_b200: B200-native (sm_100a) apg-sgm dense stereo matching.

Python front-end mirroring the reference binding (python/apg_sgm/__init__.py and
python/src/binding.cpp of WildEgoLee/apg-sgm): the same StereoSession / StereoResult /
PipelineStats / StageTiming classes, enums, keyword arguments and error behaviour, running on the
CUDA engine in libapg_sgm_b200.so through its C-ABI (include/apg_sgm/c_api.h and
include/apg_sgm_cuda.h).  `Engine` exposes the configuration-level engine used by tests, the
benchmark and the batched/served forms.
"""
from __future__ import annotations

import ctypes as C
import enum
import threading

import numpy as np

from . import _lib as _lib_mod
from ._lib import ImageView, PipelineConfig, SessionOptions, lib

__version__ = "1.0.0"


class QualityMode(enum.IntEnum):
    Fast = 0
    Balanced = 1
    HighQuality = 2


class HierarchicalFallback(enum.IntEnum):
    """HierarchicalFallback (include/apg_sgm/config.hpp:68-72): the range of a pixel whose 2x2
    coarse neighbourhood has no valid disparity."""
    NearestValid = 0
    FullRange = 1
    ExpandedRadius = 2


class VolumeBackend(enum.IntEnum):
    Auto = 0
    Dense = 1
    Packed = 2
    CUDA = 3


class MemoryPolicy(enum.IntEnum):
    ReleasePerFrame = 0
    BoundedReuse = 1


class StatusCode(enum.IntEnum):
    Ok = 0
    EmptyInput = 1
    SizeMismatch = 2
    InvalidDisparityRange = 3
    InvalidConfig = 4
    UnsupportedBackend = 5
    ResourceLimitExceeded = 6
    AllocationFailure = 7
    InternalError = 8


class InvalidReason(enum.IntEnum):
    Valid = 0
    Occlusion = 1
    Mismatch = 2
    LowConfidence = 3
    OutOfRange = 4


_STAGES = ["aux_ms", "prior_ms", "cost_ms", "cross_ms", "right_wta_ms", "sgm_ms", "wta_ms",
           "confidence_ms", "refine_ms", "post_ms", "total_ms"]


class StageTiming:
    """Per-stage device times in ms (include/apg_sgm/pipeline_stats.hpp:10-22).  The WTA is
    fused into the last SGM sweep, so its time is part of sgm_ms and wta_ms is 0."""

    def __init__(self, ms=None):
        ms = ms if ms is not None else [0.0] * 11
        for k, v in zip(_STAGES, ms):
            setattr(self, k, float(v))

    def to_dict(self):
        return {k: getattr(self, k) for k in _STAGES}

    def __repr__(self):
        return f"<StageTiming total={self.total_ms}ms (sgm={self.sgm_ms}ms, cost={self.cost_ms}ms)>"


class PipelineStats:
    """PipelineStats (include/apg_sgm/pipeline_stats.hpp:24-142) for one frame."""

    def __init__(self):
        self.timing = StageTiming()
        self.peak_workspace_bytes = 0
        self.retained_workspace_bytes = 0
        self.cost_bytes = 0
        self.estimated_peak_bytes = 0
        self.frame_allocation_count = 0
        self.frame_reuse_count = 0
        self.allocation_count = 0
        self.reuse_count = 0
        self.valid_disparity_ratio = 0.0
        self.reliable_ratio = 0.0
        self.unreliable_ratio = 0.0
        self.refine_changed_ratio = 0.0
        self.lr_fail_ratio = 0.0
        self.valid_pixels = self.reliable_pixels = self.unreliable_pixels = 0
        self.refine_changed_pixels = self.lr_fail_pixels = self.prior_support_count = 0
        self.mean_search_width = self.mean_geometry_width = 0.0
        self.effective_threads = 0
        self.requested_threads = 0
        self.requested_backend = "Auto"
        self.resolved_backend = "CUDA"
        self.memory_policy = "ReleasePerFrame"

    def to_dict(self):
        return {
            "timing": self.timing.to_dict(),
            "peak_workspace_bytes": self.peak_workspace_bytes,
            "retained_workspace_bytes": self.retained_workspace_bytes,
            "valid_disparity_ratio": self.valid_disparity_ratio,
            "reliable_ratio": self.reliable_ratio,
            "unreliable_ratio": self.unreliable_ratio,
            "effective_threads": self.effective_threads,
            "resolved_backend": self.resolved_backend,
            "memory_policy": self.memory_policy,
        }

    def __repr__(self):
        return (f"<PipelineStats total={self.timing.total_ms}ms valid_ratio={self.valid_disparity_ratio} "
                f"peak_ws_mb={self.peak_workspace_bytes / (1024.0 * 1024.0)}>")


class StereoResult:
    def __init__(self, disparity, confidence, reliable_mask, invalid_reason, stats):
        self._d, self._c, self._r, self._i = disparity, confidence, reliable_mask, invalid_reason
        self._stats = stats

    width = property(lambda self: 0 if self._d is None else self._d.shape[1])
    height = property(lambda self: 0 if self._d is None else self._d.shape[0])
    empty = property(lambda self: self._d is None or self._d.size == 0)
    stats = property(lambda self: self._stats)
    disparity = property(lambda self: self._d)
    confidence = property(lambda self: self._c)
    reliable_mask = property(lambda self: self._r)
    invalid_reason = property(lambda self: self._i)

    def __repr__(self):
        return f"<apg_sgm.StereoResult {self.width}x{self.height} valid={'False' if self.empty else 'True'}>"


def config_from_mode(mode=QualityMode.Balanced, max_disparity=128, min_disparity=0, **overrides) -> PipelineConfig:
    """PipelineConfig::from_mode (src/config.cpp:5-45) plus field overrides."""
    c = PipelineConfig()
    lib().apgcu_config_from_mode(int(mode), int(max_disparity), C.byref(c))
    c.min_disparity = int(min_disparity)
    c.volume_backend = int(VolumeBackend.CUDA)
    for k, v in overrides.items():
        if not hasattr(c, k):
            raise AttributeError(f"unknown configuration field {k!r}")
        setattr(c, k, v)
    return c


def _image_view(a, name):
    """Validate and wrap an HxW or HxWxC uint8 array (make_image_view, binding.cpp:37-119)."""
    if not isinstance(a, np.ndarray):
        a = np.asarray(a)
    if a.dtype != np.uint8:
        raise TypeError(f"{name} must have dtype uint8 (got format '{a.dtype.char}')")
    if a.ndim not in (2, 3):
        raise ValueError(f"{name} must be 2D (H, W) or 3D (H, W, C), got {a.ndim}D")
    h, w = a.shape[:2]
    c = 1 if a.ndim == 2 else a.shape[2]
    if h <= 0 or w <= 0 or h > 2**31 - 1 or w > 2**31 - 1:
        raise ValueError(f"{name} dimensions must be strictly positive and fit within INT_MAX ({w}x{h})")
    if c not in (1, 3):
        raise ValueError(f"{name} must have 1 or 3 channels, got {c}")
    zero_copy = a.strides[1] == c and (a.ndim == 2 or a.strides[2] == 1) and a.strides[0] >= w * c
    if not zero_copy:
        a = np.ascontiguousarray(a)
    v = ImageView(a.ctypes.data, w, h, a.strides[0], c)
    return v, a


def _parse(value, enum_cls, table, what):
    if value is None:
        return None
    if isinstance(value, str):
        s = value.lower()
        if s not in table:
            first = {}
            for k, v in table.items():
                first.setdefault(v, k)
            valid = ", ".join(f"'{k}'" for k in first.values())
            raise ValueError(f"Unrecognized {what} '{s}'. Valid: {valid}")
        return table[s]
    return enum_cls(int(value))


_MODES = {"fast": QualityMode.Fast, "balanced": QualityMode.Balanced, "high_quality": QualityMode.HighQuality,
          "hq": QualityMode.HighQuality, "highquality": QualityMode.HighQuality}
_BACKENDS = {"auto": VolumeBackend.Auto, "dense": VolumeBackend.Dense, "packed": VolumeBackend.Packed,
             "cuda": VolumeBackend.CUDA}
_FALLBACKS = {"nearest_valid": HierarchicalFallback.NearestValid, "nearest": HierarchicalFallback.NearestValid,
              "full_range": HierarchicalFallback.FullRange, "full": HierarchicalFallback.FullRange,
              "expanded_radius": HierarchicalFallback.ExpandedRadius, "expanded": HierarchicalFallback.ExpandedRadius}
_POLICIES = {"bounded_reuse": MemoryPolicy.BoundedReuse, "boundedreuse": MemoryPolicy.BoundedReuse,
             "reuse": MemoryPolicy.BoundedReuse, "release_per_frame": MemoryPolicy.ReleasePerFrame,
             "release": MemoryPolicy.ReleasePerFrame, "releaseperframe": MemoryPolicy.ReleasePerFrame}


class _ResultPool:
    """apg_result_t objects (each owns one page-locked block holding a frame's four maps) lent to
    the arrays that StereoSession.process returns.  A result goes back to the pool when the last
    array viewing it is gone, so in a loop that drops each frame's arrays before the next call the
    same one or two blocks serve every frame, with no allocation and no copy; results kept alive by
    the caller simply make the pool lend a new block.  No lock: a lease may be released by the
    garbage collector on any thread at any allocation, even inside take() or give_back(), and the
    list's append and pop are atomic on their own."""

    def __init__(self, keep: int = 4):
        self._free = []
        self._keep = keep
        self._closed = False

    def take(self):
        try:
            return self._free.pop()
        except IndexError:
            pass
        r = lib().apg_result_create()
        if not r:
            raise MemoryError("apg_result_create failed")
        return r

    def give_back(self, r):
        if not self._closed and len(self._free) < self._keep:
            self._free.append(r)
            if not self._closed:
                return
            try:  # closed meanwhile: close() may have missed it
                self._free.remove(r)
            except ValueError:
                return
        lib().apg_result_destroy(r)

    def close(self):
        self._closed = True
        while True:
            try:
                r = self._free.pop()
            except IndexError:
                break
            lib().apg_result_destroy(r)


class _ResultLease:
    """Holds one pooled apg_result_t while any array views its maps."""

    __slots__ = ("_pool", "_r")

    def __init__(self, pool: _ResultPool, r):
        self._pool, self._r = pool, r

    def __del__(self):
        try:
            self._pool.give_back(self._r)
        except Exception:
            pass


def _result_views(res, lease, w: int, h: int):
    """The four maps of a filled apg_result_t as numpy arrays over its page-locked block (no copy);
    the block stays lent to them (through `lease`) until the last of them is gone."""
    L = lib()
    n = w * h
    pd = L.apg_result_get_disparity(res, None, None)
    ptrs = (pd, L.apg_result_get_confidence(res, None, None), L.apg_result_get_invalid_reason(res, None, None),
            L.apg_result_get_reliable_mask(res, None, None))
    offs = [p - pd for p in ptrs]
    if any(o < 0 or o > 9 * n for o in offs):
        raise RuntimeError("result maps are not one block")
    block = (C.c_uint8 * (10 * n)).from_address(pd)
    block._lease = lease
    disp = np.frombuffer(block, np.float32, n, offs[0]).reshape(h, w)
    conf = np.frombuffer(block, np.float32, n, offs[1]).reshape(h, w)
    reason = np.frombuffer(block, np.uint8, n, offs[2]).reshape(h, w)
    rel = np.frombuffer(block, np.uint8, n, offs[3]).reshape(h, w)
    return disp, conf, rel, reason


class StereoSession:
    """Stateful streaming matcher session (PyStereoSession, binding.cpp:147-357).

    Calls on one session are serialised by a lock; independent sessions run concurrently
    (ctypes releases the GIL for the duration of every library call).  process() returns arrays
    that view a page-locked result block the device copies landed in (binding.cpp:483-531 returns
    views over a fresh per-call result in the same way): no copy, and the block is not reused
    while any of them is alive."""

    def __init__(self, mode="balanced", threads=0, max_disparity=128, min_disparity=0, backend="auto",
                 memory_policy="release_per_frame", max_retained_bytes=0, hierarchical=False, hierarchical_radius=4,
                 hierarchical_fallback=None, adaptive_radius=False, confidence_threshold=0.5, expanded_radius=8,
                 config: PipelineConfig | None = None):
        qm = _parse(mode, QualityMode, _MODES, "mode")
        if qm is None:
            qm = QualityMode.Balanced
        be = _parse(backend, VolumeBackend, _BACKENDS, "backend")
        mp = _parse(memory_policy, MemoryPolicy, _POLICIES, "memory_policy")
        if mp is None:
            mp = MemoryPolicy.ReleasePerFrame
        if config is None:
            cfg = config_from_mode(qm, max_disparity if max_disparity > 0 else 128)
            if min_disparity != 0:
                cfg.min_disparity = int(min_disparity)
            if max_disparity > 0:
                cfg.max_disparity = int(max_disparity)
            if threads > 0:
                cfg.num_threads = int(threads)
        else:
            cfg = config
        if be is not None:
            cfg.volume_backend = int(be)
        if hierarchical:
            # binding.cpp:200-223
            cfg.hier_enable = 1
            cfg.hier_radius = int(hierarchical_radius)
            cfg.hier_adaptive_radius = 1 if adaptive_radius else 0
            cfg.hier_confidence_threshold = float(confidence_threshold)
            cfg.hier_expanded_radius = int(expanded_radius)
            fb = _parse(hierarchical_fallback, HierarchicalFallback, _FALLBACKS, "hierarchical_fallback")
            if fb is not None:
                cfg.hier_fallback = int(fb)
        err = _validate_config(cfg)
        if err:
            raise RuntimeError(err)
        self._cfg = cfg
        self._policy = mp
        self._requested_backend = "Auto" if be in (None, VolumeBackend.Auto) else be.name
        self._h = lib().apgcu_session_create_config(C.byref(cfg), int(mp), C.c_size_t(int(max_retained_bytes)))
        if not self._h:
            raise RuntimeError("failed to create session")
        self._results = _ResultPool()
        self._mu = threading.Lock()

    @property
    def config(self) -> PipelineConfig:
        return self._cfg

    def process(self, left, right) -> StereoResult:
        lv, la = _image_view(left, "left")
        rv, ra = _image_view(right, "right")
        if lv.width != rv.width or lv.height != rv.height:
            raise ValueError(f"Left and right images must have identical dimensions ({lv.width}x{lv.height} vs "
                             f"{rv.width}x{rv.height})")
        if lv.channels != rv.channels:
            raise ValueError(f"Left and right images must have matching channel counts ({lv.channels} vs "
                             f"{rv.channels})")
        L = lib()
        res = self._results.take()
        lease = _ResultLease(self._results, res)
        with self._mu:
            rc = L.apg_session_process(self._h, C.byref(lv), C.byref(rv), res)
            if rc != 0:
                msg = L.apg_session_get_last_error(self._h).decode()
                raise RuntimeError(f"Stereo processing failed [{rc}]: {msg}")
            disp, conf, rel, reason = _result_views(res, lease, lv.width, lv.height)
            stats = self._stats(lv.width, lv.height)
        return StereoResult(disp, conf, rel, reason, stats)

    compute = process

    def set_tuning(self, key: str, value: int):
        """Engine tuning key for this session's frames (Engine.set_tuning's keys)."""
        rc = lib().apgcu_session_set_tuning(self._h, key.encode(), int(value))
        if rc != 0:
            raise ValueError(f"invalid tuning {key}={value}")

    def _stats(self, w: int, h: int) -> PipelineStats:
        """PipelineStats of the last frame; the pixel counters come from the device
        (apgcu_session_get_frame_counts), the ratios are float32 divisions as in
        src/pipeline.cpp:701-707."""
        ms = (C.c_double * 11)()
        cnt = (C.c_size_t * 4)()
        fc = (C.c_ulonglong * 8)()
        lib().apgcu_session_get_stats(self._h, ms, cnt)
        lib().apgcu_session_get_frame_counts(self._h, fc)
        s = PipelineStats()
        s.timing = StageTiming(list(ms))
        s.frame_allocation_count = s.allocation_count = int(cnt[0])
        s.frame_reuse_count = s.reuse_count = int(cnt[1])
        s.peak_workspace_bytes = int(cnt[2])
        s.retained_workspace_bytes = int(cnt[3])
        n = w * h
        D = self._cfg.D
        s.cost_bytes = n * D * 2
        s.estimated_peak_bytes = int(lib().apgcu_session_estimate_bytes(self._h, w, h, 1))
        (s.valid_pixels, s.reliable_pixels, s.unreliable_pixels, s.refine_changed_pixels, s.lr_fail_pixels,
         s.prior_support_count) = (int(v) for v in fc[:6])
        s.mean_search_width = fc[6] / n if n else 0.0
        s.mean_geometry_width = fc[7] / n if n else 0.0
        if n:
            nf = np.float32(n)
            s.valid_disparity_ratio = float(np.float32(s.valid_pixels) / nf)
            s.reliable_ratio = float(np.float32(s.reliable_pixels) / nf)
            s.unreliable_ratio = float(np.float32(s.unreliable_pixels) / nf)
            s.refine_changed_ratio = float(np.float32(s.refine_changed_pixels) / nf)
            s.lr_fail_ratio = float(np.float32(s.lr_fail_pixels) / nf)
        s.requested_threads = s.effective_threads = int(self._cfg.num_threads)
        s.requested_backend = self._requested_backend
        s.resolved_backend = "CUDA"
        s.memory_policy = self._policy.name
        return s

    def reset(self):
        with self._mu:
            lib().apg_session_reset(self._h)

    @property
    def frame_count(self):
        return int(lib().apg_session_get_frame_count(self._h))

    @property
    def total_time_ms(self):
        return float(lib().apg_session_get_total_time_ms(self._h))

    @property
    def average_time_ms(self):
        n = self.frame_count
        return self.total_time_ms / n if n else 0.0

    @property
    def allocated_bytes(self):
        return int(lib().apg_session_get_allocated_bytes(self._h))

    @property
    def last_error(self):
        return lib().apg_session_get_last_error(self._h).decode()

    @property
    def hierarchical_enabled(self) -> bool:
        return bool(self._cfg.hier_enable)

    @property
    def hierarchical_radius(self) -> int:
        return int(self._cfg.hier_radius)

    @property
    def adaptive_radius(self) -> bool:
        return bool(self._cfg.hier_adaptive_radius)

    @property
    def hierarchical_telemetry(self) -> dict:
        """HierarchicalTelemetry of the last frame (src/hierarchical_stereo.hpp:36-42); all zero
        without hierarchical mode or for frames under 32 x 32."""
        return _hier_dict(lib().apgcu_session_hier_telemetry, self._h)

    def __repr__(self):
        # PyStereoSession::repr, binding.cpp:335-351
        r = (f"<apg_sgm.StereoSession frames={self.frame_count} avg_time_ms={self.average_time_ms} "
             f"allocated_bytes={self.allocated_bytes}")
        if self._cfg.hier_enable:
            r += f" hierarchical=True (R={self._cfg.hier_radius}"
            if self._cfg.hier_adaptive_radius:
                r += f", adaptive_R={self._cfg.hier_expanded_radius}@{self._cfg.hier_confidence_threshold:.2f}"
            r += ")"
        return r + ">"

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                lib().apg_session_destroy(self._h)
                self._h = None
            if getattr(self, "_results", None):
                self._results.close()  # results still lent to live arrays are freed when those go
        except Exception:
            pass


def _validate_config(cfg: PipelineConfig) -> str:
    """validate_config (src/pipeline.cpp:171-213); returns the message or ''."""
    if cfg.max_disparity <= cfg.min_disparity:
        return "max_disparity must be strictly greater than min_disparity"
    if cfg.cost_max < 0 or cfg.cost_max > 65535:
        return "cost_max out of valid uint16 representation range [0, 65535]"
    if cfg.P1 < 0:
        return "SGM P1 penalty must be non-negative"
    if cfg.P2_base <= cfg.P1:
        return "SGM P2_base must be strictly greater than P1"
    if cfg.grad_t1 < 0 or cfg.grad_t2 < cfg.grad_t1:
        return "SGM gradient thresholds must satisfy 0 <= grad_t1 <= grad_t2"
    if cfg.prior_enable and cfg.prior_search_radius < 0:
        return "prior search_radius must be non-negative"
    if cfg.refine_enable and cfg.refine_iterations < 0:
        return "refine iterations must be non-negative"
    if cfg.hier_enable:
        if cfg.volume_backend == VolumeBackend.Dense:
            return "hierarchical mode requires Auto or Packed backend"
        if cfg.hier_radius <= 0:
            return "hierarchical radius must be strictly positive"
        if cfg.hier_scale != 2:
            return "hierarchical scale currently supports only 2"
        if cfg.hier_adaptive_radius:
            if cfg.hier_expanded_radius < cfg.hier_radius:
                return "hierarchical expanded_radius cannot be less than radius"
            if not (0.0 <= cfg.hier_confidence_threshold <= 1.0):
                return "hierarchical confidence_threshold must be between 0.0 and 1.0"
    return ""


_HIER_KEYS = ("avg_states_per_pixel", "coarse_valid_ratio", "fallback_pixel_ratio", "full_range_pixel_ratio",
              "coarse_time_ms")


def _hier_dict(fn, handle) -> dict:
    v = (C.c_double * 6)()
    rc = fn(handle, v)
    if rc != 0:
        raise RuntimeError(f"hierarchical telemetry failed [{rc}]")
    d = dict(zip(_HIER_KEYS, list(v)[:5]))
    d["coarse_pass"] = bool(v[5])
    return d


DUMPS = ["left_gray", "left_gx", "left_gy", "right_gray", "right_gx", "right_gy", "census_left", "census_right",
         "range_min", "range_max", "cost_raw", "cost_agg", "sgm_sum", "disp_wta", "best", "second", "disp_right",
         "confidence", "reliable", "reason_conf", "disp_refined", "disp_lr", "reason", "disp_fill", "disparity",
         "d_prior"]
_DUMP_DT = {"left_gray": np.uint8, "left_gx": np.uint8, "left_gy": np.uint8, "right_gray": np.uint8,
            "right_gx": np.uint8, "right_gy": np.uint8, "census_left": np.uint32, "census_right": np.uint32,
            "range_min": np.int16, "range_max": np.int16, "cost_raw": np.uint16, "cost_agg": np.uint16,
            "sgm_sum": np.uint16, "reliable": np.uint8, "reason_conf": np.uint8, "reason": np.uint8}

DEBUG_RAW_COST, DEBUG_KEEP_SUM, DEBUG_NO_FUSION, DEBUG_PROFILE = 1, 2, 4, 8


class Engine:
    """Configuration-level engine (apgcu_engine_*): host or device-resident processing, stage
    dumps and per-stage device times."""

    def __init__(self, config: PipelineConfig, device: int = 0, stream: int | None = None, debug: int = 0):
        err = _validate_config(config)
        if err:
            raise RuntimeError(err)
        self.config = config
        self._h = lib().apgcu_engine_create(C.byref(config), int(device), C.c_void_p(stream) if stream else None)
        if not self._h:
            raise RuntimeError("apgcu_engine_create failed (configuration outside the CUDA backend's limits?)")
        if debug:
            lib().apgcu_engine_set_debug(self._h, int(debug))
        self._shape = None

    def process(self, left, right) -> dict:
        lv, la = _image_view(left, "left")
        rv, ra = _image_view(right, "right")
        if lv.stride != rv.stride:
            la, ra = np.ascontiguousarray(la), np.ascontiguousarray(ra)
            lv, rv = _image_view(la, "left")[0], _image_view(ra, "right")[0]
        h, w = lv.height, lv.width
        out = {"disparity": np.empty((h, w), np.float32), "confidence": np.empty((h, w), np.float32),
               "invalid_reason": np.empty((h, w), np.uint8), "reliable_mask": np.empty((h, w), np.uint8)}
        rc = lib().apgcu_engine_process(self._h, lv.data, rv.data, w, h, lv.stride, lv.channels,
                                        out["disparity"].ctypes.data, out["confidence"].ctypes.data,
                                        out["invalid_reason"].ctypes.data, out["reliable_mask"].ctypes.data)
        if rc != 0:
            raise RuntimeError(f"processing failed [{rc}]: {self.last_error}")
        self._shape = (h, w)
        return out

    def process_device(self, d_left: int, d_right: int, width: int, height: int, stride: int, channels: int,
                       d_disp: int = 0, d_conf: int = 0, d_reason: int = 0, d_reliable: int = 0):
        rc = lib().apgcu_engine_process_device(self._h, d_left, d_right, width, height, stride, channels,
                                               d_disp or None, d_conf or None, d_reason or None, d_reliable or None)
        if rc != 0:
            raise RuntimeError(f"processing failed [{rc}]: {self.last_error}")
        self._shape = (height, width)

    def sync(self):
        rc = lib().apgcu_engine_sync(self._h)
        if rc != 0:
            raise RuntimeError(self.last_error)

    def supports(self):
        """The prior's selected supports of the last pair in the reference's order
        (PipelineBuffers::supports): x, y (int32), disparity, confidence (float32) arrays."""
        n = lib().apgcu_engine_supports(self._h, None, None, None, None, 0)
        if n < 0:
            raise RuntimeError(self.last_error)
        x, y = np.empty(n, np.int32), np.empty(n, np.int32)
        d, c = np.empty(n, np.float32), np.empty(n, np.float32)
        lib().apgcu_engine_supports(self._h, x.ctypes.data, y.ctypes.data, d.ctypes.data, c.ctypes.data, n)
        return x, y, d, c

    def hier_telemetry(self) -> dict:
        """HierarchicalTelemetry of the last pair (apgcu_engine_hier_telemetry)."""
        return _hier_dict(lib().apgcu_engine_hier_telemetry, self._h)

    @property
    def stream(self) -> int:
        return int(lib().apgcu_engine_stream(self._h) or 0)

    def dump(self, name: str) -> np.ndarray:
        h, w = self._shape
        D = self.config.D
        idx = DUMPS.index(name)
        if name in ("cost_raw", "cost_agg", "sgm_sum"):
            a = np.empty((h, w, D), np.uint16)
        elif name in ("census_left", "census_right") and self.config.census_type == 0:
            a = np.empty((h, w), np.uint64)
        else:
            a = np.empty((h, w), _DUMP_DT.get(name, np.float32))
        rc = lib().apgcu_engine_dump(self._h, idx, a.ctypes.data, a.nbytes)
        if rc != 0:
            raise RuntimeError(f"dump {name} failed [{rc}]: {self.last_error}")
        return a

    def stage_times(self) -> dict:
        ms = (C.c_double * 11)()
        lib().apgcu_engine_stage_times(self._h, ms)
        return dict(zip(_STAGES, list(ms)))

    def launch_profile(self) -> list:
        """[(kernel name, ms)] of the last pair, in launch order (needs DEBUG_PROFILE)."""
        names = (C.c_char_p * 64)()
        ms = (C.c_float * 64)()
        n = lib().apgcu_engine_launch_profile(self._h, 64, names, ms)
        return [(names[i].decode(), float(ms[i])) for i in range(n)]

    def set_debug(self, flags: int):
        lib().apgcu_engine_set_debug(self._h, int(flags))

    def set_tuning(self, key: str, value: int):
        rc = lib().apgcu_engine_set_tuning(self._h, key.encode(), int(value))
        if rc != 0:
            raise ValueError(f"invalid tuning {key}={value}")

    @property
    def allocated_bytes(self) -> int:
        return int(lib().apgcu_engine_allocated_bytes(self._h))

    def release(self):
        lib().apgcu_engine_release(self._h)

    @property
    def last_error(self) -> str:
        return lib().apgcu_engine_last_error(self._h).decode()

    def close(self):
        if getattr(self, "_h", None):
            lib().apgcu_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def kernel_launch_count() -> int:
    return int(lib().apgcu_kernel_launch_count())


StereoMetrics = _lib_mod.StereoMetricsRec
RegionMetrics = _lib_mod.RegionMetricsRec


def evaluate_stereo(est, gt, range=None, d_before_refine=None, d_after_refine=None, vis_mask=None,
                    max_valid_gt: float = 1e5, left_image=None, thresholds=None, stream=None) -> StereoMetrics:
    """evaluate_stereo (src/metrics.cpp:119-502; the support block is not part of it) on the GPU.

    est, gt: HxW float32 disparity maps; range: (range_min, range_max) int16 planes; the refine
    maps, vis_mask (uint8, >= 200 = visible) and left_image (HxW or HxWx3 uint8) are optional as in
    the reference.  thresholds: (boundary_disparity_gradient, low_texture_gradient, max_valid_gt),
    default QualityThresholds{}.  Either all arrays are numpy (host; copied in) or all are CUDA
    tensors of the current device (evaluated in place on `stream`, default the current torch
    stream).  Returns the record (attributes as StereoMetrics; .to_dict())."""
    arrays = [est, gt, None if range is None else range[0], None if range is None else range[1], d_before_refine,
              d_after_refine, vis_mask, left_image]
    present = [a for a in arrays if a is not None]
    on_device = all(hasattr(a, "is_cuda") and a.is_cuda for a in present)
    if not on_device and any(hasattr(a, "is_cuda") and a.is_cuda for a in present):
        raise ValueError("evaluate_stereo: pass all arrays on the host or all on the device")
    want = [np.float32, np.float32, np.int16, np.int16, np.float32, np.float32, np.uint8, np.uint8]
    keep, ptrs = [], []
    h, w = (int(gt.shape[0]), int(gt.shape[1]))
    for a, dt in zip(arrays, want):
        if a is None:
            ptrs.append(None)
            continue
        if on_device:
            import torch
            tdt = {np.float32: torch.float32, np.int16: torch.int16, np.uint8: torch.uint8}[dt]
            if a.dtype != tdt:
                raise TypeError(f"evaluate_stereo: expected {tdt}, got {a.dtype}")
            a = a.contiguous()
            keep.append(a)
            ptrs.append(C.c_void_p(a.data_ptr()))
        else:
            a = np.ascontiguousarray(a, dt)
            keep.append(a)
            ptrs.append(a.ctypes.data_as(C.c_void_p))
        if tuple(a.shape[:2]) != (h, w):
            raise ValueError(f"evaluate_stereo: every map must be {h}x{w}")
    lch = 0 if left_image is None else (1 if len(left_image.shape) == 2 else int(left_image.shape[2]))
    thr = None
    if thresholds is not None:
        thr = _lib_mod.QualityThresholdsRec(*[float(v) for v in thresholds])
    if on_device and stream is None:
        import torch
        stream = torch.cuda.current_stream().cuda_stream
    out = StereoMetrics()
    rc = lib().apgcu_evaluate_stereo(ptrs[0], ptrs[1], w, h, ptrs[2], ptrs[3], ptrs[4], ptrs[5], ptrs[6],
                                     C.c_float(max_valid_gt), ptrs[7], w * lch, lch,
                                     C.byref(thr) if thr is not None else None, 1 if on_device else 0,
                                     C.c_void_p(stream) if stream else None, C.byref(out))
    if rc != 0:
        raise RuntimeError(f"evaluate_stereo failed [{rc}]")
    return out


# ---- On-disk formats (src/image.cpp:62-206) ----------------------------------------------------

def _path(p) -> bytes:
    return str(p).encode()


def _io_check(rc: int, what: str, path):
    if rc != 0:
        raise OSError(f"{what} failed for {path} [{rc}]")


def load_image(path) -> np.ndarray:
    """load_image: binary PGM (HxW) or PPM (HxWx3) as uint8."""
    w, h, c = C.c_int(), C.c_int(), C.c_int()
    _io_check(lib().apgcu_image_info(_path(path), C.byref(w), C.byref(h), C.byref(c)), "load_image", path)
    a = np.empty((h.value, w.value, c.value) if c.value > 1 else (h.value, w.value), np.uint8)
    _io_check(lib().apgcu_load_image(_path(path), a.ctypes.data, a.nbytes, C.byref(w), C.byref(h), C.byref(c)),
              "load_image", path)
    return a


def save_pgm(path, img):
    a = np.ascontiguousarray(img, np.uint8)
    if a.ndim != 2:
        raise ValueError("save_pgm takes a single-channel HxW image")
    _io_check(lib().apgcu_save_pgm(_path(path), a.ctypes.data, a.shape[1], a.shape[0]), "save_pgm", path)


def save_pgm16(path, disp):
    a = np.ascontiguousarray(disp, np.int16)
    _io_check(lib().apgcu_save_pgm16(_path(path), a.ctypes.data, a.shape[1], a.shape[0]), "save_pgm16", path)


def save_disparity_preview(path, disp, dmax: float):
    a = np.ascontiguousarray(disp, np.float32)
    _io_check(lib().apgcu_save_disparity_preview(_path(path), a.ctypes.data, a.shape[1], a.shape[0],
                                                 C.c_float(dmax)), "save_disparity_preview", path)


def load_pfm(path) -> np.ndarray:
    """load_pfm: HxW float32 (channel 0 of a colour PFM), top row first."""
    w, h, c = C.c_int(), C.c_int(), C.c_int()
    _io_check(lib().apgcu_pfm_info(_path(path), C.byref(w), C.byref(h), C.byref(c)), "load_pfm", path)
    a = np.empty((h.value, w.value), np.float32)
    _io_check(lib().apgcu_load_pfm(_path(path), a.ctypes.data, a.size, C.byref(w), C.byref(h)), "load_pfm", path)
    return a


def save_pfm(path, img):
    a = np.ascontiguousarray(img, np.float32)
    _io_check(lib().apgcu_save_pfm(_path(path), a.ctypes.data, a.shape[1], a.shape[0]), "save_pfm", path)


class Loader:
    """Pair loader (apgcu_loader_*): worker threads read (left, right) image files into page-locked
    buffers the loader recycles.  wait() lends the pair as numpy views of those buffers, valid until
    release()."""

    def __init__(self, threads: int = 4):
        self._h = lib().apgcu_loader_create(int(threads))
        if not self._h:
            raise RuntimeError("apgcu_loader_create failed")

    def submit(self, left_path, right_path) -> int:
        t = C.c_ulonglong()
        rc = lib().apgcu_loader_submit(self._h, _path(left_path), _path(right_path), C.byref(t))
        if rc != 0:
            raise RuntimeError(f"loader submit failed [{rc}]")
        return t.value

    def wait(self, ticket: int):
        p = _lib_mod.LoadedPair()
        rc = lib().apgcu_loader_wait(self._h, int(ticket), C.byref(p))
        if rc != 0:
            raise OSError(f"loading pair {ticket} failed [{rc}]")
        shape = (p.height, p.width, p.channels) if p.channels > 1 else (p.height, p.width)
        n = p.width * p.height * p.channels
        views = []
        for ptr in (p.left, p.right):
            buf = (C.c_uint8 * n).from_address(ptr)
            views.append(np.frombuffer(buf, np.uint8).reshape(shape))
        return views[0], views[1]

    def release(self, ticket: int):
        lib().apgcu_loader_release(self._h, int(ticket))

    @property
    def pinned_bytes(self) -> int:
        return int(lib().apgcu_loader_pinned_bytes(self._h))

    def close(self):
        if getattr(self, "_h", None):
            lib().apgcu_loader_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def serve_files(server: "Server", pairs, mode=QualityMode.Balanced, max_disparity=128, min_disparity=0,
                loader: Loader = None, depth: int = 16, out_pool=None):
    """Runs (left_path, right_path) pairs through `server`, reading ahead with a Loader: up to
    `depth` pairs are read or in flight at once, each pair's page-locked images go to the server as
    they are, and a pair's buffers return to the loader when its request completes.  out_pool
    (optional): a list of at least `depth` caller-owned result dicts (see Server.submit) reused in
    turn.  Yields (index, outputs, latency_ms) in submission order."""
    own = loader is None
    ld = loader or Loader()
    pairs = list(pairs)
    tickets, inflight = {}, []
    nxt = 0
    try:
        while nxt < len(pairs) and len(tickets) < depth:
            tickets[nxt] = ld.submit(*pairs[nxt])
            nxt += 1
        for i in range(len(pairs)):
            if i in tickets:
                lt = tickets.pop(i)
                left, right = ld.wait(lt)
                out = out_pool[i % len(out_pool)] if out_pool else None
                inflight.append((i, lt, server.submit(left, right, mode=mode, max_disparity=max_disparity,
                                                      min_disparity=min_disparity, out=out)))
            while inflight and (len(inflight) >= depth or i == len(pairs) - 1):
                j, lt, st = inflight.pop(0)
                o, lat = server.wait(st)
                ld.release(lt)
                if nxt < len(pairs):
                    tickets[nxt] = ld.submit(*pairs[nxt])
                    nxt += 1
                yield j, o, lat
    finally:
        for j, lt, st in inflight:
            try:
                server.wait(st)
            except Exception:
                pass
            ld.release(lt)
        if own:
            ld.close()


# ---- Experimental scopes (src/subpixel_estimator.hpp, src/inpaint_internal.hpp) -----------------

class SubpixelMethod(enum.IntEnum):
    Legacy = 0
    CurvGate = 1
    ConfGate = 2
    Stabilized = 3


class InpaintMethod(enum.IntEnum):
    Legacy = 0
    ShadowReclass = 1


_SUBPIXEL = {"legacy": SubpixelMethod.Legacy, "a": SubpixelMethod.Legacy, "curv_gate": SubpixelMethod.CurvGate,
             "curv": SubpixelMethod.CurvGate, "b": SubpixelMethod.CurvGate, "conf_gate": SubpixelMethod.ConfGate,
             "conf": SubpixelMethod.ConfGate, "c": SubpixelMethod.ConfGate, "stabilized": SubpixelMethod.Stabilized,
             "stab": SubpixelMethod.Stabilized, "d": SubpixelMethod.Stabilized}
_INPAINT = {"legacy": InpaintMethod.Legacy, "a": InpaintMethod.Legacy, "shadow_reclass": InpaintMethod.ShadowReclass,
            "shadow": InpaintMethod.ShadowReclass, "c": InpaintMethod.ShadowReclass}


def _get_experimental():
    sm, sp, im, ig = C.c_int(), C.c_float(), C.c_int(), C.c_int()
    lib().apgcu_get_experimental(C.byref(sm), C.byref(sp), C.byref(im), C.byref(ig))
    return sm.value, sp.value, im.value, ig.value


def _get_telemetry_flags():
    a, b = C.c_int(), C.c_int()
    lib().apgcu_get_experimental_telemetry(C.byref(a), C.byref(b))
    return a.value, b.value


class SubpixelTelemetry:
    """SubpixelTelemetry (src/subpixel_estimator.hpp:50-118): this thread's counters."""

    def __init__(self, rec):
        for k, _ in rec._fields_:
            v = getattr(rec, k)
            setattr(self, k, list(v) if k == "delta_buckets" else v)

    def applied_ratio(self) -> float:
        return self.applied_pixels / self.candidate_pixels if self.candidate_pixels else 0.0

    def clamped_ratio(self) -> float:
        return self.clamped_count / self.applied_pixels if self.applied_pixels else 0.0

    def mean_abs_delta(self) -> float:
        return self.sum_abs_delta / self.applied_pixels if self.applied_pixels else 0.0

    def percentile_abs_delta(self, q: float) -> float:
        if self.applied_pixels == 0:
            return 0.0
        import math
        target = int(math.ceil(float(np.float32(np.float32(q) * np.float32(self.applied_pixels)))))
        acc = 0
        for i, c in enumerate(self.delta_buckets):
            acc += c
            if acc >= target:
                return float(np.float32(np.float32(i + 0.5) * np.float32(0.01)))
        return 0.5

    def p50_abs_delta(self) -> float:
        return self.percentile_abs_delta(0.50)

    def p95_abs_delta(self) -> float:
        return self.percentile_abs_delta(0.95)


class InpaintTelemetry:
    """InpaintTelemetry (src/inpaint_internal.hpp:65-163): this thread's counters."""

    _ROUTES = ["none", "occ_both_min", "occ_left_only", "occ_right_only", "mismatch_color_horiz",
               "mismatch_color_vert", "mismatch_prior", "mismatch_lerp", "mismatch_left_only",
               "mismatch_right_only", "remained_invalid"]

    def __init__(self, rec):
        for k, _ in rec._fields_:
            v = getattr(rec, k)
            setattr(self, k, list(v) if k in ("route_counts", "run_length_buckets") else v)

    def route(self, name: str) -> int:
        return self.route_counts[self._ROUTES.index(name)]

    def total_filled_pixels(self) -> int:
        rem = self.route_counts[10]
        return self.total_invalid_pixels - rem if self.total_invalid_pixels > rem else 0

    def fill_ratio(self) -> float:
        return self.total_filled_pixels() / self.total_invalid_pixels if self.total_invalid_pixels else 0.0

    def occ_filled_pixels(self) -> int:
        return self.route_counts[1] + self.route_counts[2] + self.route_counts[3]

    def occ_unfilled_pixels(self) -> int:
        a = self.classified_occ_pixels + self.reclassified_shadow_pixels
        return a - self.occ_filled_pixels() if a > self.occ_filled_pixels() else 0

    def mismatch_native_filled_pixels(self) -> int:
        return sum(self.route_counts[4:10])

    def mismatch_filled_pixels(self) -> int:
        return self.mismatch_native_filled_pixels() + self.reclassified_shadow_pixels

    def mismatch_unfilled_pixels(self) -> int:
        f = self.mismatch_filled_pixels()
        return self.classified_mismatch_pixels - f if self.classified_mismatch_pixels > f else 0


def _telemetry():
    sp, ip = _lib_mod.SubpixelTelemetryRec(), _lib_mod.InpaintTelemetryRec()
    lib().apgcu_get_telemetry(C.byref(sp), C.byref(ip))
    return sp, ip


class ExperimentalSubpixelScope:
    """ExperimentalSubpixelScope (src/subpixel_estimator.hpp:130-155): within the `with` block, every
    frame this thread runs uses `method` (parse_subpixel_method's names or SubpixelMethod) with
    `param` (<= 0: the method's default) for the WTA and right-image sub-pixel step; with
    collect_telemetry the WTA's counters accumulate into current_telemetry() (reset on entry).  The
    previous scope returns on exit."""

    def __init__(self, method=SubpixelMethod.Legacy, param: float = 0.0, collect_telemetry: bool = False):
        m = _parse(method, SubpixelMethod, _SUBPIXEL, "subpixel method")
        self.method, self.param = (SubpixelMethod.Legacy if m is None else m), float(param)
        self.collect = bool(collect_telemetry)

    def __enter__(self):
        self._prev = _get_experimental()
        self._prev_tel = _get_telemetry_flags()
        _, _, im, ig = self._prev
        lib().apgcu_set_experimental(int(self.method), C.c_float(self.param), im, ig)
        lib().apgcu_set_experimental_telemetry(int(self.collect), _get_telemetry_flags()[1])
        if self.collect:
            lib().apgcu_reset_telemetry(1, 0)
        return self

    def __exit__(self, *exc):
        sm, sp, _, _ = self._prev
        _, _, im, ig = _get_experimental()
        lib().apgcu_set_experimental(sm, C.c_float(sp), im, ig)
        lib().apgcu_set_experimental_telemetry(self._prev_tel[0], _get_telemetry_flags()[1])
        return False

    @staticmethod
    def current_telemetry() -> SubpixelTelemetry:
        return SubpixelTelemetry(_telemetry()[0])


class ExperimentalInpaintScope:
    """ExperimentalInpaintScope (src/inpaint_internal.hpp, src/postprocess.cpp:42-53): within the
    `with` block every frame this thread runs fills holes with `method` (Legacy or ShadowReclass)
    and `max_gap` (Legacy at 32 keeps the configuration's max_fill_gap); with collect_telemetry the
    fill's counters accumulate into current_telemetry() (reset on entry)."""

    def __init__(self, method=InpaintMethod.Legacy, max_gap: int = 32, collect_telemetry: bool = False):
        m = _parse(method, InpaintMethod, _INPAINT, "inpaint method")
        self.method, self.max_gap = (InpaintMethod.Legacy if m is None else m), int(max_gap)
        self.collect = bool(collect_telemetry)

    def __enter__(self):
        self._prev = _get_experimental()
        self._prev_tel = _get_telemetry_flags()
        sm, sp, _, _ = self._prev
        lib().apgcu_set_experimental(sm, C.c_float(sp), int(self.method), self.max_gap)
        lib().apgcu_set_experimental_telemetry(_get_telemetry_flags()[0], int(self.collect))
        if self.collect:
            lib().apgcu_reset_telemetry(0, 1)
        return self

    def __exit__(self, *exc):
        _, _, im, ig = self._prev
        sm, sp, _, _ = _get_experimental()
        lib().apgcu_set_experimental(sm, C.c_float(sp), im, ig)
        lib().apgcu_set_experimental_telemetry(_get_telemetry_flags()[0], self._prev_tel[1])
        return False

    @staticmethod
    def current_telemetry() -> InpaintTelemetry:
        return InpaintTelemetry(_telemetry()[1])


SupportMetrics = _lib_mod.SupportMetricsRec


def evaluate_supports(supports, gt, vis_mask=None, max_valid_gt: float = 1e5, cell_size: int = 16) -> SupportMetrics:
    """evaluate_supports (src/metrics.cpp:8-124) on the GPU: supports = (x, y, disparity[, ...])
    arrays (Engine.supports()), gt HxW float32, vis_mask HxW uint8 (>= 200 visible) or None."""
    x, y, d = (np.ascontiguousarray(a, t) for a, t in zip(supports[:3], (np.int32, np.int32, np.float32)))
    gt = np.ascontiguousarray(gt, np.float32)
    h, w = gt.shape
    vis = None if vis_mask is None else np.ascontiguousarray(vis_mask, np.uint8)
    out = SupportMetrics()
    rc = lib().apgcu_evaluate_supports(x.ctypes.data, y.ctypes.data, d.ctypes.data, len(x), gt.ctypes.data, w, h,
                                       None if vis is None else vis.ctypes.data, C.c_float(max_valid_gt),
                                       int(cell_size), 0, None, C.byref(out))
    if rc != 0:
        raise RuntimeError(f"evaluate_supports failed [{rc}]")
    return out


def workspace_bytes(config: PipelineConfig, width: int, height: int) -> int:
    return int(lib().apgcu_workspace_bytes(C.byref(config), int(width), int(height)))


__all__ = ["QualityMode", "HierarchicalFallback", "VolumeBackend", "MemoryPolicy", "StatusCode", "InvalidReason", "StageTiming",
           "PipelineStats", "StereoResult", "StereoSession", "PipelineConfig", "config_from_mode", "Engine",
           "kernel_launch_count", "workspace_bytes", "evaluate_stereo", "StereoMetrics", "RegionMetrics",
           "evaluate_supports", "SupportMetrics", "load_image", "save_pgm", "save_pgm16", "save_disparity_preview", "load_pfm", "save_pfm", "Loader",
           "serve_files", "SubpixelMethod", "InpaintMethod", "ExperimentalSubpixelScope", "ExperimentalInpaintScope",
           "SubpixelTelemetry", "InpaintTelemetry",
           "__version__"]



_OUT_DTYPES = {"disparity": np.float32, "confidence": np.float32, "invalid_reason": np.uint8,
               "reliable_mask": np.uint8}


def _result_arrays(h: int, w: int, out=None) -> dict:
    """The four result maps of one pair: `out` (caller-owned, checked) or fresh arrays."""
    if out is None:
        return {k: np.empty((h, w), dt) for k, dt in _OUT_DTYPES.items()}
    for k, dt in _OUT_DTYPES.items():
        a = out[k]
        if a.shape != (h, w) or a.dtype != dt or not a.flags.c_contiguous or not a.flags.writeable:
            raise ValueError(f"out[{k!r}] must be a writeable C-contiguous {np.dtype(dt).name} array of shape {(h, w)}")
    return out

class Batch:
    """Batched form (apgcu_batch_*): many pairs of uneven sizes and disparity ranges per call.

    Pairs of equal size and range form a bucket; a bucket's pairs run their per-pixel stages
    concurrently and share one persistent SGM launch per phase, replayed from a cached CUDA graph.
    Each pair's outputs equal those of Engine.process for that pair alone."""

    def __init__(self, config: PipelineConfig, device: int = 0, **options):
        err = _validate_config(config)
        if err:
            raise RuntimeError(err)
        self.config = config
        self._h = lib().apgcu_batch_create(C.byref(config), int(device))
        if not self._h:
            raise RuntimeError("apgcu_batch_create failed")
        for k, v in options.items():
            self.set_option(k, v)

    def set_option(self, key: str, value: int):
        if lib().apgcu_batch_set_option(self._h, key.encode(), int(value)) != 0:
            raise ValueError(f"invalid batch option {key}={value}")

    def process(self, pairs, out=None) -> list:
        """pairs: iterable of (left, right) or (left, right, max_disparity) host arrays.  Returns one
        dict of disparity / confidence / invalid_reason / reliable_mask per pair: `out[i]` when a
        list of caller-owned dicts is given (page-locked ones take the device copies directly),
        else new arrays."""
        keep, outs = [], []
        arr = (_lib_mod.Pair * len(pairs))()
        for i, p in enumerate(pairs):
            left, right = p[0], p[1]
            dmax = int(p[2]) if len(p) > 2 else 0
            lv, la = _image_view(left, "left")
            rv, ra = _image_view(right, "right")
            if lv.stride != rv.stride:
                la, ra = np.ascontiguousarray(la), np.ascontiguousarray(ra)
                lv, rv = _image_view(la, "left")[0], _image_view(ra, "right")[0]
            h, w = lv.height, lv.width
            o = _result_arrays(h, w, out[i] if out is not None else None)
            keep += [la, ra]
            outs.append(o)
            arr[i] = _lib_mod.Pair(lv.data, rv.data, w, h, lv.stride, lv.channels, dmax,
                                   o["disparity"].ctypes.data, o["confidence"].ctypes.data,
                                   o["invalid_reason"].ctypes.data, o["reliable_mask"].ctypes.data)
        rc = lib().apgcu_batch_process(self._h, len(pairs), arr, 0)
        if rc != 0:
            raise RuntimeError(f"batch processing failed [{rc}]: {self.last_error}")
        return outs

    def process_device(self, pairs) -> None:
        """pairs: list of _lib.Pair records holding device pointers (inputs and outputs)."""
        arr = (_lib_mod.Pair * len(pairs))(*pairs)
        rc = lib().apgcu_batch_process(self._h, len(pairs), arr, 1)
        if rc != 0:
            raise RuntimeError(f"batch processing failed [{rc}]: {self.last_error}")

    @property
    def last_error(self) -> str:
        return lib().apgcu_batch_last_error(self._h).decode()

    @property
    def allocated_bytes(self) -> int:
        return int(lib().apgcu_batch_allocated_bytes(self._h))

    @property
    def last_time_ms(self) -> float:
        """Device time of the last call (start event to the latest bucket end)."""
        return float(lib().apgcu_batch_last_time_ms(self._h))

    def release(self):
        lib().apgcu_batch_release(self._h)

    def close(self):
        if getattr(self, "_h", None):
            lib().apgcu_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_MODE_VALUE = {"fast": 0, "balanced": 1, "high_quality": 2, "hq": 2}


class Server:
    """Served form (apgcu_server_*): a request loop with continuous batching.

    `slots` requests run at once, each on a device-resident engine of its (mode, size, range)
    borrowed from a pool; engine workspaces are admitted against an HBM budget.  submit() returns
    at once; wait() returns the outputs and the submission-to-completion latency in ms."""

    def __init__(self, device: int = 0, hbm_budget_gb: float = 120.0, slots: int = 4):
        self._h = lib().apgcu_server_create(int(device), int(hbm_budget_gb * (1 << 30)), int(slots))
        if not self._h:
            raise RuntimeError("apgcu_server_create failed (no CUDA device?)")
        self._pending = {}

    def submit(self, left, right, mode=QualityMode.Balanced, max_disparity=128, min_disparity=0,
               outputs: bool = True, out: dict = None) -> int:
        """Queues one pair; `out` (optional) holds caller-owned C-contiguous result arrays (disparity and
        confidence float32, invalid_reason and reliable_mask uint8, each height x width) that the
        request writes instead of new ones.  They must stay alive and untouched until wait()."""
        lv, la = _image_view(left, "left")
        rv, ra = _image_view(right, "right")
        if lv.stride != rv.stride:
            la, ra = np.ascontiguousarray(la), np.ascontiguousarray(ra)
            lv, rv = _image_view(la, "left")[0], _image_view(ra, "right")[0]
        h, w = lv.height, lv.width
        o = _result_arrays(h, w, out) if (out is not None or outputs) else None
        ptr = (lambda k: o[k].ctypes.data) if o else (lambda k: None)
        req = _lib_mod.Request(int(_MODE_VALUE.get(mode, mode)), int(min_disparity), int(max_disparity),
                               lv.data, rv.data, w, h, lv.stride, lv.channels, ptr("disparity"), ptr("confidence"),
                               ptr("invalid_reason"), ptr("reliable_mask"))
        t = C.c_ulonglong()
        rc = lib().apgcu_server_submit(self._h, C.byref(req), C.byref(t))
        if rc != 0:
            raise RuntimeError(f"submit failed [{rc}]")
        self._pending[t.value] = (la, ra, o)
        return t.value

    def wait(self, ticket: int):
        lat = C.c_double()
        rc = lib().apgcu_server_wait(self._h, int(ticket), C.byref(lat))
        _, _, o = self._pending.pop(ticket)
        if rc != 0:
            raise RuntimeError(f"request failed [{rc}]: {lib().apgcu_server_last_error(self._h).decode()}")
        return o, lat.value

    def reserve(self, width: int, height: int, mode=QualityMode.Balanced, max_disparity=128, min_disparity=0,
                channels: int = 1, count: int = 1):
        """Warm pool: `count` idle device-resident engines for requests of this mode, size and range."""
        req = _lib_mod.Request(int(_MODE_VALUE.get(mode, mode)), int(min_disparity), int(max_disparity), None, None,
                               int(width), int(height), int(width) * int(channels), int(channels),
                               None, None, None, None)
        rc = lib().apgcu_server_reserve(self._h, C.byref(req), int(count))
        if rc != 0:
            raise RuntimeError(f"reserve failed [{rc}]")

    def stats(self) -> dict:
        c = (C.c_ulonglong * 4)()
        b = (C.c_size_t * 2)()
        lib().apgcu_server_stats(self._h, c, b)
        return {"completed": c[0], "failed": c[1], "evictions": c[2], "peak_in_flight": c[3],
                "reserved_bytes": b[0], "peak_reserved_bytes": b[1],
                "budget_bytes": int(lib().apgcu_server_budget(self._h))}

    def close(self):
        if getattr(self, "_h", None):
            lib().apgcu_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
