"""Hierarchical coarse-to-fine search range: oracle pins and host logic (no GPU).

The oracle's restatement (orc_hier_range in oracle/apg_oracle.c) is checked against the
reference's own output: the committed fixtures (tests/golden/hier_fixtures.npz, written by
tests/golden/make_golden_hier.py from the reference build) and, where oracle/_ref is built, live
runs of the reference on further inputs.  The configuration checks mirror
tests/test_hierarchical.cpp (test_hierarchical_validation) and python/tests/test_bindings.py
(test_hierarchical_session_lifecycle, test_hierarchical_invalid_parameters).
"""
from pathlib import Path

import numpy as np
import pytest

from helpers import same_bits, synth

FIX = Path(__file__).resolve().parent / "golden" / "hier_fixtures.npz"
MAPS = ("disparity", "confidence", "invalid_reason", "reliable_mask")


def _cases():
    if not FIX.exists():
        return []
    with np.load(FIX) as z:
        return [str(c) for c in z["cases"]]


@pytest.mark.parametrize("case", _cases())
def test_oracle_matches_hier_fixtures(case, O):
    z = np.load(FIX)
    cfg = O.config_from_record(z[f"{case}/config"].tobytes())
    L, R = z[f"{case}/left"], z[f"{case}/right"]
    got = O.hier_range(cfg, L, R)
    for k in ("range_min", "range_max", "d_prior"):
        assert same_bits(got[k], z[f"{case}/{k}"]), (case, k)
    t = z[f"{case}/telemetry"]
    assert got["ran"] == int(t[4])
    assert got["telemetry"]["avg_states_per_pixel"] == t[0]
    assert got["telemetry"]["coarse_valid_ratio"] == t[1]
    assert got["telemetry"]["fallback_pixel_ratio"] == t[2]
    assert got["telemetry"]["full_range_pixel_ratio"] == t[3]
    out = O.pipeline(cfg, L, R)
    assert out["status"] == 0
    for k in MAPS:
        assert same_bits(out[k], z[f"{case}/{k}"]), (case, k)


LIVE = [
    # mode, w, h, dmax, dmin, patch, overrides
    (1, 130, 70, 40, 0, 0.3, {}),
    (0, 64, 64, 24, 0, 0.0, {"hier_fallback": 2}),
    (1, 75, 45, 32, 10, 0.25, {"hier_coarse_fill_holes": 0, "hier_fallback": 0}),
    (2, 90, 60, 40, -6, 0.2, {"hier_adaptive_radius": 1, "hier_expanded_radius": 12, "hier_confidence_threshold": 0.7}),
    (1, 33, 32, 16, 0, 0.0, {}),
    (1, 31, 64, 16, 0, 0.0, {}),
]


@pytest.mark.parametrize("case", LIVE, ids=[f"live{i}" for i in range(len(LIVE))])
def test_oracle_matches_reference_live(case, O):
    if not O.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    mode, w, h, dmax, dmin, patch, over = case
    cfg = O.config(mode, dmax, dmin, hier_enable=1, **over)
    L, R = synth(w, h, dmax, patch=patch, seed=w * 7 + h)
    ref = O.ref_hier_dump(cfg, L, R)
    assert ref["status"] == 0
    got = O.hier_range(cfg, L, R)
    for k in ("range_min", "range_max", "d_prior"):
        assert same_bits(got[k], ref[k]), k
    assert got["ran"] == ref["ran"]
    for k, v in ref["telemetry"].items():
        assert got["telemetry"][k] == v, k
    out = O.pipeline(cfg, L, R)
    for k in MAPS:
        assert same_bits(out[k], ref[k]), k


def test_coarse_config_restatement(O):
    """hierarchical_stereo.cpp:172-182: half bounds (C++ truncating division), no prior/refine."""
    for d0, dmax, want in [(0, 128, (0, 64)), (0, 129, (0, 65)), (-24, 40, (0, 20)), (7, 9, (3, 5)),
                           (-64, -10, (0, 1)), (5, 6, (2, 3))]:
        cfg = O.config(2, dmax, d0, hier_enable=1, hier_coarse_cross_agg=0, hier_coarse_fill_holes=0)
        c = O.hier_coarse_config(cfg)
        assert (c.min_disparity, c.max_disparity) == want
        assert (c.prior_enable, c.refine_enable, c.agg_enable, c.subpixel, c.lr_check) == (0, 0, 0, 1, 1)
        assert (c.median_radius, c.max_fill_gap, c.hier_enable, c.paths) == (1, 0, 0, 8)


def test_hierarchical_validation(apg):
    """tests/test_hierarchical.cpp:192-235 through the library's own validation."""
    base = apg.config_from_mode(1, 32, hier_enable=1)
    e = apg.Engine  # construction validates; no frame is processed

    def bad(**kw):
        c = apg.config_from_mode(1, 32, hier_enable=1, **kw)
        with pytest.raises(RuntimeError):
            e(c)

    bad(volume_backend=int(apg.VolumeBackend.Dense))
    bad(hier_radius=0)
    bad(hier_radius=-2)
    for sc in (1, 3, 4):
        bad(hier_scale=sc)
    bad(hier_adaptive_radius=1, hier_expanded_radius=2)
    bad(hier_adaptive_radius=1, hier_confidence_threshold=-0.1)
    bad(hier_adaptive_radius=1, hier_confidence_threshold=1.5)
    for be in (apg.VolumeBackend.Auto, apg.VolumeBackend.Packed, apg.VolumeBackend.CUDA):
        c = apg.config_from_mode(1, 32, hier_enable=1, volume_backend=int(be))
        e(c).close()
    # without adaptive radius the expanded radius and threshold are not checked
    e(apg.config_from_mode(1, 32, hier_enable=1, hier_expanded_radius=1, hier_confidence_threshold=3.0)).close()
    e(base).close()


def test_hierarchical_session_lifecycle(apg):
    s = apg.StereoSession(mode="balanced", max_disparity=64, hierarchical=True, hierarchical_radius=4,
                          hierarchical_fallback="nearest_valid")
    assert s.hierarchical_enabled is True
    assert s.hierarchical_radius == 4
    assert s.adaptive_radius is False
    assert "hierarchical=True (R=4)" in repr(s)
    s2 = apg.StereoSession(mode="balanced", max_disparity=32, hierarchical=True, hierarchical_radius=4,
                           adaptive_radius=True, confidence_threshold=0.5, expanded_radius=8)
    assert s2.adaptive_radius is True
    assert "adaptive_R=8@0.50" in repr(s2)
    plain = apg.StereoSession(mode="balanced", max_disparity=32)
    assert plain.hierarchical_enabled is False and "hierarchical" not in repr(plain)
    for name, want in (("full", 1), ("FULL_RANGE", 1), ("expanded", 2), ("nearest", 0)):
        s3 = apg.StereoSession(mode="fast", max_disparity=32, hierarchical=True, hierarchical_fallback=name)
        assert s3.config.hier_fallback == want
    # the fallback and radii are only applied with hierarchical=True (binding.cpp:200)
    s4 = apg.StereoSession(mode="fast", max_disparity=32, hierarchical_radius=0)
    assert s4.hierarchical_enabled is False


def test_hierarchical_invalid_parameters(apg):
    with pytest.raises(RuntimeError, match="hierarchical radius must be strictly positive"):
        apg.StereoSession(mode="fast", max_disparity=32, hierarchical=True, hierarchical_radius=0)
    with pytest.raises(RuntimeError, match="expanded_radius cannot be less than radius"):
        apg.StereoSession(mode="fast", max_disparity=32, hierarchical=True, adaptive_radius=True, expanded_radius=2)
    with pytest.raises(RuntimeError, match="confidence_threshold must be between 0.0 and 1.0"):
        apg.StereoSession(mode="fast", max_disparity=32, hierarchical=True, adaptive_radius=True,
                          confidence_threshold=1.5)
    with pytest.raises(RuntimeError, match="requires Auto or Packed backend"):
        apg.StereoSession(mode="fast", max_disparity=32, backend="dense", hierarchical=True)
    with pytest.raises(ValueError, match="Unrecognized hierarchical_fallback 'bogus'"):
        apg.StereoSession(mode="fast", max_disparity=32, hierarchical=True, hierarchical_fallback="bogus")


def test_hierarchical_workspace_estimate(apg):
    """The workspace estimate covers the half-size engine for frames of 32 x 32 and more."""
    plain = apg.config_from_mode(1, 64)
    hier = apg.config_from_mode(1, 64, hier_enable=1)
    small = apg.workspace_bytes(hier, 40, 20)
    assert small >= apg.workspace_bytes(plain, 40, 20)
    big_p, big_h = apg.workspace_bytes(plain, 320, 240), apg.workspace_bytes(hier, 320, 240)
    assert big_h > big_p
    # the coarse engine works on a quarter of the pixels with half the range: well under half
    assert big_h - big_p < big_p // 2
