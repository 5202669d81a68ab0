"""Full-size parity against the reference's own StereoSession (Packed backend, oracle/_ref).

The benchmark workloads at their real sizes, through both public entry points of this library
(the engine and the C-API session), compared bit for bit with the reference CPU pipeline
(StereoMatcher::compute_status, src/pipeline.cpp:337-397) on the same seeded synthetic pairs:

* 1280x720 D128 Balanced: the size and mode the bit-exactness target names;
* 1920x1080 D256 HighQuality: 8,160 prior cells with the default budget of 4,000 supports, so the
  stratified selection (src/prior_estimator.cpp:112-168) binds; 34 refiner bands in one
  cooperative launch, with the shared-memory window and with the L1 form; the vertical
  aggregation with per-pixel ranges at Dp 256 over 1080 rows;
* 1242x375 D192 Balanced (the KITTI-sized configuration), 640x480 D64 Balanced,
  1280x720 D128 Fast, 1920x1080 D256 Balanced and 1280x720 D128 Balanced in hierarchical mode.

Every final map (disparity, confidence, invalid_reason, reliable_mask) is compared by bit pattern
(tolerance 0, max |delta| = 0, floats included), and so are the PipelineStats counters and ratios.
"""
import numpy as np
import pytest

from helpers import same_bits

pytestmark = pytest.mark.gpu

MAPS = ("disparity", "confidence", "invalid_reason", "reliable_mask")
COUNTS = ("valid_pixels", "reliable_pixels", "unreliable_pixels", "refine_changed_pixels", "prior_support_count")
RATIOS = ("valid_disparity_ratio", "reliable_ratio", "unreliable_ratio", "refine_changed_ratio", "lr_fail_ratio",
          "mean_search_width", "mean_geometry_width")

# name: (mode, PairSpec args, configuration overrides, engine tuning)
CASES = {
    "balanced_1280x720_d128": (1, (1280, 720, 128, 12, 0, 120, 0.0), {}, {}),
    "highquality_1920x1080_d256": (2, (1920, 1080, 256, 16, 0, 240, 0.2), {}, {}),
    "highquality_1920x1080_d256_l1_window": (2, (1920, 1080, 256, 16, 0, 240, 0.2), {}, {"refine_window": 1}),
    "balanced_1242x375_d192": (1, (1242, 375, 192, 12, 0, 180, 0.0), {}, {}),
    "balanced_640x480_d64": (1, (640, 480, 64, 8, 4, 60, 0.0), {}, {}),
    "fast_1280x720_d128": (0, (1280, 720, 128, 12, 0, 120, 0.0), {}, {}),
    "balanced_1920x1080_d256": (1, (1920, 1080, 256, 16, 0, 240, 0.0), {}, {}),
    "balanced_1280x720_d128_hierarchical": (1, (1280, 720, 128, 12, 0, 120, 0.0), {"hier_enable": 1}, {}),
}

_REF_CACHE = {}


def _pair(spec_args):
    from apg_sgm_b200 import synthetic as S
    L, R, _ = S.make_pair(S.PairSpec(*spec_args), S.SEED_BASE)
    return L, R


def _reference(O, name, mode, spec_args, over, L, R):
    """The reference session's frame for (mode, spec, overrides), cached across the two entry
    points (the tuning variants share their reference frame)."""
    key = (mode, spec_args, tuple(sorted(over.items())))
    if key not in _REF_CACHE:
        sess = O.RefSession(O.config(mode, spec_args[2], volume_backend=2, **over))
        ref = sess.process(L, R)
        sess.close()
        assert ref["status"] == 0, f"{name}: reference status {ref['status']}"
        _REF_CACHE[key] = ref
    return _REF_CACHE[key]


def _need_ref(O):
    if not O.ref_available():
        pytest.skip("oracle/_ref (the reference build) is not present")


def _check_maps(name, got, ref):
    for k in MAPS:
        a, b = got[k], ref[k]
        if not same_bits(a, b):
            bad = np.argwhere(a != b)
            i = tuple(int(v) for v in bad[0]) if len(bad) else None
            pytest.fail(f"{name}: {k} differs from the reference at {len(bad)} pixels; first {i}: "
                        f"gpu={a[i] if i else None} reference={b[i] if i else None}")


@pytest.mark.parametrize("name", sorted(CASES))
def test_engine_matches_reference_session(name, O, apg):
    _need_ref(O)
    mode, spec_args, over, tune = CASES[name]
    L, R = _pair(spec_args)
    cfg = apg.config_from_mode(mode, spec_args[2], **over)
    eng = apg.Engine(cfg)
    for k, v in tune.items():
        eng.set_tuning(k, v)
    got = eng.process(L, R)
    eng.close()
    _check_maps(name, got, _reference(O, name, mode, spec_args, over, L, R))


@pytest.mark.parametrize("name", sorted(CASES))
def test_session_matches_reference_session(name, O, apg):
    """apg_session_process (the reference's C entry point) over the CUDA engine: maps and
    PipelineStats (src/pipeline.cpp:650-707) equal the reference session's."""
    _need_ref(O)
    mode, spec_args, over, tune = CASES[name]
    L, R = _pair(spec_args)
    sess = apg.StereoSession(mode={0: "fast", 1: "balanced", 2: "high_quality"}[mode], max_disparity=spec_args[2],
                             memory_policy="bounded_reuse", hierarchical=bool(over.get("hier_enable")))
    for k, v in tune.items():
        sess.set_tuning(k, v)
    res = sess.process(L, R)
    ref = _reference(O, name, mode, spec_args, over, L, R)
    _check_maps(name, {k: getattr(res, k) for k in MAPS}, ref)
    st, rs = res.stats, ref["stats"]
    for k in COUNTS:
        assert getattr(st, k) == int(rs[k]), (name, k, getattr(st, k), rs[k])
    for k in RATIOS:
        assert getattr(st, k) == rs[k], (name, k, getattr(st, k), rs[k])
    if mode == 2:
        # 1920x1080 has 120 x 68 = 8,160 cells of 16x16: the default 4,000-support budget binds
        assert rs["prior_support_count"] == 4000


def test_highquality_1080p_second_frame_same(O, apg):
    """A second HighQuality frame through the same session (arena, refiner state and draw-table
    positions reused) gives the same maps as the reference."""
    _need_ref(O)
    mode, spec_args, over, _ = CASES["highquality_1920x1080_d256"]
    L, R = _pair(spec_args)
    sess = apg.StereoSession(mode="high_quality", max_disparity=spec_args[2], memory_policy="bounded_reuse")
    sess.process(L, R)
    res = sess.process(L, R)
    _check_maps("hq second frame", {k: getattr(res, k) for k in MAPS},
                _reference(O, "hq", mode, spec_args, over, L, R))
