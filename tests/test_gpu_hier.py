"""Hierarchical coarse-to-fine search range on the GPU against the reference and the oracle.

The device path (hier.cu: 2x2 downsample and per-pixel range step around a half-size engine run
on the same stream) must give bit-identical range planes, guiding disparities, telemetry and
final maps:
  * against the reference's own outputs frozen in tests/golden/hier_fixtures.npz;
  * against the oracle (orc_hier_range + orc_pipeline) on further shapes: odd sizes, negative and
    positive minimum disparities, all three fallbacks, the adaptive radius, coarse aggregation and
    fill switched off, HighQuality with the refiner, RGB input;
and through every entry point that takes a configuration: the engine (host and device buffers),
the session (streaming with BoundedReuse, as tests/test_hierarchical.cpp:237-282) and the batch.
At 1280 x 720 the size-independent properties are checked instead: ranges inside the geometric
bounds, telemetry consistent with the frame counters.
"""
from pathlib import Path

import numpy as np
import pytest

from helpers import same_bits, synth, to_oracle

pytestmark = pytest.mark.gpu

FIX = Path(__file__).resolve().parent / "golden" / "hier_fixtures.npz"
MAPS = ("disparity", "confidence", "invalid_reason", "reliable_mask")
PLANES = ("range_min", "range_max", "d_prior")


def _fixture_cases():
    if not FIX.exists():
        return []
    with np.load(FIX) as z:
        return [str(c) for c in z["cases"]]


def _run(apg, cfg, L, R, **tuning):
    e = apg.Engine(cfg)
    for k, v in tuning.items():
        e.set_tuning(k, v)
    out = e.process(L, R)
    planes = {k: e.dump(k) for k in PLANES}
    tel = e.hier_telemetry()
    e.close()
    return out, planes, tel


@pytest.mark.parametrize("case", _fixture_cases())
def test_hier_matches_reference_fixtures(case, O, apg):
    z = np.load(FIX)
    ocfg = O.config_from_record(z[f"{case}/config"].tobytes())
    cfg = apg.PipelineConfig.from_buffer_copy(bytes(ocfg))
    L, R = z[f"{case}/left"], z[f"{case}/right"]
    out, planes, tel = _run(apg, cfg, L, R)
    for k in PLANES:
        assert same_bits(planes[k], z[f"{case}/{k}"]), (case, k)
    for k in MAPS:
        assert same_bits(out[k], z[f"{case}/{k}"]), (case, k)
    t = z[f"{case}/telemetry"]
    assert tel["coarse_pass"] == bool(t[4])
    assert (tel["avg_states_per_pixel"], tel["coarse_valid_ratio"], tel["fallback_pixel_ratio"],
            tel["full_range_pixel_ratio"]) == tuple(t[:4])


CASES = [
    # name, mode, w, h, dmax, dmin, patch, overrides
    ("balanced_320x200_d64", 1, 320, 200, 64, 0, 0.2, {}),
    ("balanced_odd_333x201_d96", 1, 333, 201, 96, 0, 0.25, {}),
    ("fast_256x96_d128", 0, 256, 96, 128, 0, 0.2, {}),
    ("fast_nocross_200x120_d64", 0, 200, 120, 64, 0, 0.2, {"hier_coarse_cross_agg": 0}),
    ("hq_240x160_d64", 2, 240, 160, 64, 0, 0.2, {}),
    ("hq_adaptive_181x97_d48", 2, 181, 97, 48, 0, 0.3,
     {"hier_adaptive_radius": 1, "hier_expanded_radius": 10, "hier_confidence_threshold": 0.6}),
    ("balanced_full_nofill_160x120_d64_d0_8", 1, 160, 120, 64, 8, 0.3,
     {"hier_fallback": 1, "hier_coarse_fill_holes": 0}),
    ("balanced_expanded_nofill_150x90_d48", 1, 150, 90, 48, 0, 0.3,
     {"hier_fallback": 2, "hier_coarse_fill_holes": 0, "hier_radius": 2}),
    ("balanced_neg_dmin_160x96", 1, 160, 96, 40, -24, 0.2, {}),
    ("balanced_d256_400x64", 1, 400, 64, 256, 0, 0.2, {}),
    ("census64_160x96", 1, 160, 96, 48, 0, 0.2, {"census_type": 0}),
    ("path8_radius1_128x64", 1, 128, 64, 32, 0, 0.2, {"paths": 8, "hier_radius": 1}),
    ("tiny_fallback_31x40", 1, 31, 40, 16, 0, 0.0, {}),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_hier_matches_oracle(case, O, apg):
    name, mode, w, h, dmax, dmin, patch, over = case
    cfg = apg.config_from_mode(mode, dmax, dmin, hier_enable=1, **over)
    L, R = synth(w, h, dmax, patch=patch, seed=w + 3 * h)
    if name.startswith("fast_256"):
        L, R = np.repeat(L[..., None], 3, 2), np.repeat(R[..., None], 3, 2)  # RGB input
    out, planes, tel = _run(apg, cfg, L, R)
    ocfg = to_oracle(O, cfg)
    want = O.hier_range(ocfg, L, R)
    for k in PLANES:
        assert same_bits(planes[k], want[k]), (name, k)
    assert tel["coarse_pass"] == bool(want["ran"])
    for k, v in want["telemetry"].items():
        assert tel[k] == v, (name, k)
    ref = O.pipeline(ocfg, L, R)
    assert ref["status"] == 0
    for k in MAPS:
        assert same_bits(out[k], ref[k]), (name, k)


@pytest.mark.parametrize("mode,dmax", [(1, 96), (0, 64), (2, 64)])
def test_hier_cost_kernels_agree(apg, mode, dmax):
    """The pixel-run and column-tile cost kernels over the hierarchical ranges (both passes)."""
    cfg = apg.config_from_mode(mode, dmax, hier_enable=1)
    L, R = synth(300, 120, dmax, patch=0.2, seed=11)
    a, pa, _ = _run(apg, cfg, L, R, cost_kernel=0)
    b, pb, _ = _run(apg, cfg, L, R, cost_kernel=1)
    for k in MAPS:
        assert same_bits(a[k], b[k]), k
    for k in PLANES:
        assert same_bits(pa[k], pb[k]), k


def test_hier_device_buffers(apg):
    import torch
    cfg = apg.config_from_mode(1, 64, hier_enable=1)
    L, R = synth(192, 128, 64, patch=0.2, seed=12)
    e = apg.Engine(cfg)
    want = e.process(L, R)
    dl, dr = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
    outs = {"disparity": torch.empty((128, 192), dtype=torch.float32, device="cuda"),
            "confidence": torch.empty((128, 192), dtype=torch.float32, device="cuda"),
            "invalid_reason": torch.empty((128, 192), dtype=torch.uint8, device="cuda"),
            "reliable_mask": torch.empty((128, 192), dtype=torch.uint8, device="cuda")}
    torch.cuda.synchronize()
    e.process_device(dl.data_ptr(), dr.data_ptr(), 192, 128, 192, 1, outs["disparity"].data_ptr(),
                     outs["confidence"].data_ptr(), outs["invalid_reason"].data_ptr(), outs["reliable_mask"].data_ptr())
    e.sync()
    e.close()
    for k in MAPS:
        assert same_bits(outs[k].cpu().numpy(), want[k]), k


def test_session_streaming_hierarchical(apg):
    """tests/test_hierarchical.cpp:237-282: retained workspace stable over 20 frames; reset frees it."""
    L, R = synth(64, 64, 32, seed=13)
    s = apg.StereoSession(mode="fast", max_disparity=32, memory_policy="bounded_reuse", hierarchical=True,
                          hierarchical_radius=4)
    first = None
    prev = None
    for f in range(20):
        res = s.process(L, R)
        assert not res.empty
        if f == 0:
            prev = s.allocated_bytes
            assert prev > 0
            first = res
        else:
            assert s.allocated_bytes == prev
            for k in ("disparity", "confidence"):
                assert same_bits(getattr(res, k), getattr(first, k)), k
    assert s.frame_count == 20
    tel = s.hierarchical_telemetry
    assert tel["coarse_pass"] and 0.0 < tel["avg_states_per_pixel"] < 32.0
    assert 0.0 <= tel["coarse_valid_ratio"] <= 1.0
    s.reset()
    assert s.allocated_bytes == 0


def test_hierarchical_end_to_end_reduces_states(apg):
    """tests/test_hierarchical.cpp:30-84 on its own pattern: a known shift of 8 pixels; fewer
    states than the full range of 32, every range inside [min_disparity, max_disparity]."""
    w, h = 128, 96
    y, x = np.mgrid[0:h, 0:w]
    pat = ((x * 37 + y * 53 + (x ^ y) * 17) % 256).astype(np.uint8)
    left = pat
    right = np.zeros_like(pat)
    xr = x - 8
    ok = (xr >= 0) & (xr < w)
    right[y[~ok], x[~ok]] = pat[~ok]
    right[y[ok], xr[ok]] = pat[ok]
    s = apg.StereoSession(mode="balanced", max_disparity=32, hierarchical=True, hierarchical_radius=4,
                          hierarchical_fallback="nearest_valid")
    res = s.process(left, right)
    tel = s.hierarchical_telemetry
    assert 0.0 < tel["avg_states_per_pixel"] < 32.0
    assert 0.0 <= tel["coarse_valid_ratio"] <= 1.0
    assert res.stats.mean_search_width == pytest.approx(tel["avg_states_per_pixel"])
    e = apg.Engine(apg.config_from_mode(1, 32, hier_enable=1))
    e.process(left, right)
    lo, hi = e.dump("range_min"), e.dump("range_max")
    e.close()
    assert (lo >= 0).all() and (hi <= 32).all() and (lo <= hi).all()


def test_batch_hierarchical_matches_engine(apg):
    sizes = [(160, 96, 64), (200, 120, 96), (160, 96, 64), (48, 40, 32)]
    pairs = [synth(w, h, d, patch=0.2, seed=20 + i) for i, (w, h, d) in enumerate(sizes)]
    cfg = apg.config_from_mode(1, 64, hier_enable=1)
    want = []
    for (L, R), (_, _, d) in zip(pairs, sizes):
        c = apg.config_from_mode(1, d, hier_enable=1)
        e = apg.Engine(c)
        want.append(e.process(L, R))
        e.close()
    b = apg.Batch(cfg)
    for rep in range(2):  # the second call replays the cached graphs
        got = b.process([(L, R, d) for (L, R), (_, _, d) in zip(pairs, sizes)])
        for i in range(len(sizes)):
            for k in MAPS:
                assert same_bits(got[i][k], want[i][k]), (rep, i, k)
    b.close()


def test_hier_720p_properties(apg):
    """Full size (1280 x 720, Balanced, D = 128): ranges inside [d0, min(dmax, x + 1)] per pixel
    (empty ones where the guided interval starts beyond it), guiding disparity below twice the
    coarse range end, the telemetry's mean width equal to
    the frame counters' mean search width, and far fewer states than the full range."""
    w, h, dmax = 1280, 720, 128
    L, R = synth(w, h, dmax, patch=0.1, seed=30)
    s = apg.StereoSession(mode="balanced", max_disparity=dmax, hierarchical=True)
    res = s.process(L, R)
    tel = s.hierarchical_telemetry
    assert tel["coarse_pass"]
    assert res.stats.mean_search_width == pytest.approx(tel["avg_states_per_pixel"], rel=1e-12)
    assert tel["avg_states_per_pixel"] < 0.3 * dmax
    e = apg.Engine(apg.config_from_mode(1, dmax, hier_enable=1))
    out = e.process(L, R)
    lo, hi, dp = e.dump("range_min"), e.dump("range_max"), e.dump("d_prior")
    e.close()
    x = np.arange(w)[None, :]
    assert (lo >= 0).all() and (lo <= hi).all()
    assert (hi <= np.maximum(np.minimum(dmax, x + 1), lo)).all()
    assert (dp < 2 * 64).all()
    for k in MAPS:
        assert same_bits(out[k], getattr(res, k)), k
