"""Frames with the last SGM sweep in row bands (tuning host_bands).

apgcu_engine_process, apgcu_engine_process_device and apg_session_process run the last
(bottom-up) sweep as several launches over bands of rows, carrying each chain's path values
between them, and post-process and copy out each band's finished rows while the next band sweeps.
Every case here runs the same pair with the banded path (default 6 bands, and 2, 3 and 16) and
with one sweep (host_bands=1), and compares the four maps bit for bit (a session test also the
PipelineStats counters); two cases are also compared with the oracle.  The shapes cover each
padded range the banded sweep takes (128, 192, 256; the byte volume at 256), heights that are
not a multiple of the 32-step bands, the stages between the sweep and the maps switched off one at
a time, hierarchical ranges, an experimental scope and the device-output entry point (tuning
device_bands there).
"""
import numpy as np
import pytest

from helpers import diff_report, same_bits, synth, to_oracle

MAPS = ("disparity", "confidence", "invalid_reason", "reliable_mask")

CASES = [
    # (id, mode, w, h, dmax, overrides)
    ("fast_1280x720_d128", 0, 1280, 720, 128, {}),
    ("balanced_1242x375_d192", 1, 1242, 375, 192, {}),
    ("balanced_600x301_d256_byte_volume", 1, 600, 301, 256, {}),
    ("fast_700x333_d256_byte_volume", 0, 700, 333, 256, {}),
    ("balanced_500x290_d128_no_median", 1, 500, 290, 128, {"median_radius": 0}),
    ("balanced_500x290_d128_no_lr", 1, 500, 290, 128, {"lr_check": 0}),
    ("balanced_500x290_d128_gap0", 1, 500, 290, 128, {"max_fill_gap": 0}),
    ("balanced_640x480_d128_hierarchical", 1, 640, 480, 128, {"hier_enable": 1}),
    ("balanced_512x257_d100_negative_min", 1, 512, 257, 100, {"min_disparity": -20}),
]


def _run(apg, cfg, L, R, bands):
    e = apg.Engine(cfg)
    e.set_tuning("host_bands", bands)
    out = e.process(L, R)
    e.close()
    return out


STAT_KEYS = ("valid_pixels", "reliable_pixels", "unreliable_pixels", "refine_changed_pixels", "lr_fail_pixels",
             "prior_support_count", "mean_search_width", "valid_disparity_ratio", "reliable_ratio", "lr_fail_ratio")


def _session(apg, cfg, frames, bands):
    s = apg.StereoSession(config=cfg, memory_policy="bounded_reuse")
    s.set_tuning("host_bands", bands)
    out = []
    for L, R in frames:
        r = s.process(L, R)
        out.append(({k: np.array(getattr(r, k)) for k in MAPS}, {k: getattr(r.stats, k) for k in STAT_KEYS}))
    del s
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_banded_host_path_changes_no_result(apg, case):
    _, mode, w, h, dmax, over = case
    over = dict(over)
    dmin = over.pop("min_disparity", 0)
    L, R = synth(w, h, dmax, cells=8, lo=max(dmin, 0), hi=dmax - 8, seed=71)
    cfg = apg.config_from_mode(mode, dmax, dmin, **over)
    want = _run(apg, cfg, L, R, 1)
    for bands in (0, 2, 16):
        got = _run(apg, cfg, L, R, bands)
        for k in MAPS:
            assert same_bits(got[k], want[k]), f"host_bands={bands} {k}: {diff_report(got[k], want[k])}"


@pytest.mark.gpu
@pytest.mark.parametrize("mode,w,h,dmax", [(0, 384, 300, 128), (1, 352, 289, 192)])
def test_banded_host_path_matches_oracle(apg, O, mode, w, h, dmax):
    L, R = synth(w, h, dmax, cells=6, lo=0, hi=dmax - 8, seed=72)
    cfg = apg.config_from_mode(mode, dmax)
    got = _run(apg, cfg, L, R, 0)
    want = O.pipeline(to_oracle(O, cfg), L, R)
    for k in MAPS:
        assert same_bits(got[k], want[k]), f"{k}: {diff_report(got[k], want[k])}"


@pytest.mark.gpu
def test_banded_session_frames_and_stats(apg):
    """Two frames of different sizes through one session (BoundedReuse): outputs and PipelineStats
    equal those of a session whose engine sweeps in one launch."""
    frames = [synth(1280, 720, 128, cells=12, lo=0, hi=120, seed=73), synth(800, 400, 128, cells=6, seed=74)]
    cfg = apg.config_from_mode(1, 128)
    res = {bands: _session(apg, cfg, frames, bands) for bands in (0, 1)}
    for (a, sa), (b, sb) in zip(res[0], res[1]):
        for k in MAPS:
            assert same_bits(a[k], b[k]), k
        assert sa == sb


@pytest.mark.gpu
def test_banded_under_experimental_scope(apg):
    """Under an experimental sub-pixel scope (no telemetry) the banded path keeps the scope's maps."""
    L, R = synth(640, 360, 128, cells=8, seed=75)
    cfg = apg.config_from_mode(1, 128)
    outs = []
    for bands in (0, 1):
        with apg.ExperimentalSubpixelScope(2, 0.3):
            outs.append(_run(apg, cfg, L, R, bands))
    for k in MAPS:
        assert same_bits(outs[0][k], outs[1][k]), k


def _run_device(apg, cfg, L, R, bands, frames=2):
    """apgcu_engine_process_device with torch device buffers; `frames` calls in a row into the same
    outputs (the second frame's copies must not race the first's)."""
    import torch
    h, w = L.shape[:2]
    e = apg.Engine(cfg)
    e.set_tuning("device_bands", bands)
    dl, dr = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
    outs = {"disparity": torch.full((h, w), 7.0, dtype=torch.float32, device="cuda"),
            "confidence": torch.full((h, w), 7.0, dtype=torch.float32, device="cuda"),
            "invalid_reason": torch.full((h, w), 9, dtype=torch.uint8, device="cuda"),
            "reliable_mask": torch.full((h, w), 9, dtype=torch.uint8, device="cuda")}
    torch.cuda.synchronize()
    for _ in range(frames):
        e.process_device(dl.data_ptr(), dr.data_ptr(), w, h, w, 1, outs["disparity"].data_ptr(),
                         outs["confidence"].data_ptr(), outs["invalid_reason"].data_ptr(),
                         outs["reliable_mask"].data_ptr())
    e.sync()
    e.close()
    return {k: v.cpu().numpy() for k, v in outs.items()}


@pytest.mark.gpu
@pytest.mark.parametrize("case", [CASES[0], CASES[1], CASES[3], CASES[4]], ids=lambda c: c[0])
def test_banded_device_path_changes_no_result(apg, case):
    """The device-output entry point (apgcu_engine_process_device) with the banded sweep (tuning
    device_bands; one sweep by default): maps in the caller's device buffers equal the one-sweep
    form's and the host path's."""
    _, mode, w, h, dmax, over = case
    over = dict(over)
    dmin = over.pop("min_disparity", 0)
    L, R = synth(w, h, dmax, cells=8, lo=max(dmin, 0), hi=dmax - 8, seed=76)
    cfg = apg.config_from_mode(mode, dmax, dmin, **over)
    want = _run(apg, cfg, L, R, 1)
    for bands in (0, 3, 6):
        got = _run_device(apg, cfg, L, R, bands)
        for k in MAPS:
            assert same_bits(got[k], want[k]), f"host_bands={bands} {k}: {diff_report(got[k], want[k])}"
