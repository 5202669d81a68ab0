"""Accuracy metrics (evaluate_stereo, src/metrics.cpp:119-502): the oracle's restatement against
the reference (no GPU).

Pinned by the reference's own known-answer test (tests/test_ablation.cpp:102-166, test_metrics),
by fixtures of the reference's outputs (tests/golden/metrics_fixtures.npz, written by
tests/golden/make_golden_metrics.py from the reference build) and, where oracle/_ref is built, by
live comparison on further inputs: NaN / inf / negative / out-of-bound GT, invalid estimates,
visibility values around the threshold, ranges, refine maps, 1- and 3-channel left images,
non-default thresholds.
"""
from pathlib import Path

import numpy as np
import pytest

from helpers import metric_case, same_metrics

FIX = Path(__file__).resolve().parent / "golden" / "metrics_fixtures.npz"


def _known_answer_inputs():
    gt = np.full((10, 10), 5.0, np.float32)
    gt[:, 5:] = 10.0
    est = np.full((10, 10), 5.0, np.float32)
    est[:, 5:] = 11.5
    rmin = np.zeros((10, 10), np.int16)
    rmax = np.full((10, 10), 10, np.int16)
    vis = np.full((10, 10), 255, np.uint8)
    vis[:, 5:] = 0
    return gt, est, rmin, rmax, vis


def test_reference_known_answer(O):
    """test_metrics (tests/test_ablation.cpp:102-166) on the oracle."""
    gt, est, rmin, rmax, vis = _known_answer_inputs()
    m = O.evaluate_stereo(est, gt, (rmin, rmax))
    assert abs(m.range_recall_all - 0.5) < 1e-4
    m = O.evaluate_stereo(est, gt, (rmin, rmax), vis=vis)
    assert abs(m.range_recall_visible - 1.0) < 1e-4
    before = np.full((10, 10), 5.0, np.float32)
    after = before.copy()
    before[:, 5:], after[:, 5:], est[:, 5:] = 12.0, 11.0, 10.5
    m = O.evaluate_stereo(est, gt, before=before, after=after)
    assert m.has_refine_stats
    assert abs(m.refine_epe_delta + 0.5) < 1e-4 and abs(m.post_epe_delta + 0.25) < 1e-4
    left = np.where(np.arange(10)[None, :] < 5, 100, np.arange(10)[None, :] * 20).astype(np.uint8).repeat(10, 0)
    m = O.evaluate_stereo(est, gt, (rmin, rmax), vis=vis, left=left)
    assert m.reg_all.total_pixels == m.evaluated_pixels and m.reg_all.valid_est_pixels == m.valid_pixels
    assert abs(m.reg_all.epe - m.epe) < 1e-4
    assert m.reg_noc.total_pixels + m.reg_occ.total_pixels == m.reg_all.total_pixels
    assert m.reg_boundary.total_pixels + m.reg_non_boundary.total_pixels == m.reg_all.total_pixels
    assert m.reg_low_texture.total_pixels + m.reg_high_texture.total_pixels == m.reg_all.total_pixels
    assert m.reg_low_texture.total_pixels > 0 and m.reg_high_texture.total_pixels > 0


CASES = [
    # name, w, h, seed, channels, quantised, options
    ("all_inputs_64x48", 64, 48, 1, 1, True, {}),
    ("rgb_left_75x41", 75, 41, 2, 3, True, {}),
    ("unquantised_90x33", 90, 33, 3, 1, False, {}),
    ("no_optional_40x30", 40, 30, 4, 1, True, {"range": False, "refine": False, "vis": False, "left": False}),
    ("thresholds_50x50", 50, 50, 5, 3, True, {"thresholds": (0.5, 10.0, 1e5), "max_valid_gt": 48.0}),
    ("single_row_33x1", 33, 1, 6, 1, True, {}),
    ("single_col_1x17", 1, 17, 7, 3, True, {}),
]


def run_case(f, case):
    name, w, h, seed, ch, q, opt = case
    d = metric_case(w, h, seed, ch, quantised=q)
    return f(d["est"], d["gt"], d["range"] if opt.get("range", True) else None,
             d["before"] if opt.get("refine", True) else None, d["after"] if opt.get("refine", True) else None,
             d["vis"] if opt.get("vis", True) else None, opt.get("max_valid_gt", 1e5),
             d["left"] if opt.get("left", True) else None, opt.get("thresholds"))


def _oracle(O):
    return lambda est, gt, rng, b, a, vis, mx, left, thr: O.evaluate_stereo(est, gt, rng, b, a, vis, mx, left, thr)


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_oracle_matches_reference_live(case, O):
    if not O.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    got = run_case(_oracle(O), case)
    want = run_case(lambda *a: O.evaluate_stereo(*a, reference=True), case)
    assert not same_metrics(got, want)
    assert got.evaluated_pixels > 0 or case[0].startswith("single")


def _fixture_cases():
    if not FIX.exists():
        return []
    with np.load(FIX) as z:
        return [str(c) for c in z["cases"]]


@pytest.mark.parametrize("case", _fixture_cases())
def test_oracle_matches_metric_fixtures(case, O):
    z = np.load(FIX)
    c = next(c for c in CASES if c[0] == case)
    got = run_case(_oracle(O), c)
    want = O.StereoMetricsRec.from_buffer_copy(z[f"{case}/record"].tobytes())
    assert not same_metrics(got, want)


SUPPORT_CASES = [(96, 64, 16, 11, True), (75, 41, 7, 12, False), (40, 30, 16, 13, True)]


@pytest.mark.parametrize("case", SUPPORT_CASES, ids=[f"{c[0]}x{c[1]}_cell{c[2]}" for c in SUPPORT_CASES])
def test_support_metrics_oracle_matches_reference(case, O):
    """evaluate_supports (src/metrics.cpp:8-124): supports inside and outside the frame, on invalid
    ground truth, visible or not, errors around 0.5 / 1 / 2."""
    if not O.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    w, h, cell, seed, with_vis = case
    d = metric_case(w, h, seed)
    rng = np.random.default_rng(seed)
    n = 300
    x = rng.integers(-3, w + 3, n).astype(np.int32)
    y = rng.integers(-3, h + 3, n).astype(np.int32)
    g0 = np.nan_to_num(d["gt"], nan=0.0, posinf=0.0, neginf=0.0)
    base = g0[np.clip(y, 0, h - 1), np.clip(x, 0, w - 1)]
    disp = (base + rng.choice(np.array([0.0, 0.5, 0.75, 1.0, 1.5, 2.0, 2.5, 9.0], np.float32), n)).astype(np.float32)
    vis = d["vis"] if with_vis else None
    got = O.evaluate_supports(x, y, disp, d["gt"], vis, 1e5, cell)
    want = O.evaluate_supports(x, y, disp, d["gt"], vis, 1e5, cell, reference=True)
    assert got.to_dict() == want.to_dict()
    assert got.gt_valid > 0 and got.visible > 0 and got.correct_1 > 0
    empty = O.evaluate_supports(x[:0], y[:0], disp[:0], d["gt"], vis, 1e5, cell)
    assert empty.total == 0 and empty.gt_valid == 0
