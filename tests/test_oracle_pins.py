"""Pins of the CPU oracle against the reference (no GPU needed).

1. The reference's frozen contract fingerprints (tests/test_api_contract.cpp:243-257 of the
   reference): FNV-1a64 of disparity / confidence / invalid_reason / reliable_mask for 13 cases.
2. The reference's 1-D SGM known-answer test (tests/test_synthetic.cpp:26-71).
3. Committed fixtures produced by the reference itself (tests/golden/make_golden.py).
4. When the reference build is present (oracle/_ref), a live stage-by-stage comparison.
"""
from pathlib import Path

import numpy as np
import pytest

from helpers import pattern, same_bits, synth

GOLDEN_TABLE = [
    # tag, w, h, invalid, reliable, disp, conf, invalid_hash, reliable_hash
    ("Odd_Checkerboard_Fast_Dense", 33, 27, 0, 612, 0x1710451f7eab215, 0xe61822cc0fbe3a38, 0x22081e533cd30004, 0x9ade9d63e4fcae7b),
    ("Color_Noise_Fast_Dense", 32, 24, 0, 720, 0x7e8e0fa784351325, 0x5860e8f479cbe0fd, 0x82f55cc1fd68a695, 0x9db48cb5d76242b5),
    ("Odd_Checkerboard_Fast_Packed", 33, 27, 0, 612, 0x1710451f7eab215, 0xe61822cc0fbe3a38, 0x22081e533cd30004, 0x9ade9d63e4fcae7b),
    ("Color_Noise_Fast_Packed", 32, 24, 0, 720, 0x7e8e0fa784351325, 0x5860e8f479cbe0fd, 0x82f55cc1fd68a695, 0x9db48cb5d76242b5),
    ("Odd_Checkerboard_Balanced_Dense", 33, 27, 0, 612, 0x1710451f7eab215, 0xe61822cc0fbe3a38, 0x22081e533cd30004, 0x9ade9d63e4fcae7b),
    ("Color_Noise_Balanced_Dense", 32, 24, 0, 720, 0x7e8e0fa784351325, 0x5860e8f479cbe0fd, 0x82f55cc1fd68a695, 0x9db48cb5d76242b5),
    ("Odd_Checkerboard_Balanced_Packed", 33, 27, 0, 612, 0x1710451f7eab215, 0xe61822cc0fbe3a38, 0x22081e533cd30004, 0x9ade9d63e4fcae7b),
    ("Color_Noise_Balanced_Packed", 32, 24, 0, 720, 0x7e8e0fa784351325, 0x5860e8f479cbe0fd, 0x82f55cc1fd68a695, 0x9db48cb5d76242b5),
    ("Odd_Checkerboard_HighQuality_Dense", 33, 27, 0, 612, 0x1710451f7eab215, 0xe61822cc0fbe3a38, 0x22081e533cd30004, 0x9ade9d63e4fcae7b),
    ("Color_Noise_HighQuality_Dense", 32, 24, 0, 720, 0x7e8e0fa784351325, 0x5860e8f479cbe0fd, 0x82f55cc1fd68a695, 0x9db48cb5d76242b5),
    ("Odd_Checkerboard_HighQuality_Packed", 33, 27, 0, 612, 0x1710451f7eab215, 0xe61822cc0fbe3a38, 0x22081e533cd30004, 0x9ade9d63e4fcae7b),
    ("Color_Noise_HighQuality_Packed", 32, 24, 0, 720, 0x7e8e0fa784351325, 0x5860e8f479cbe0fd, 0x82f55cc1fd68a695, 0x9db48cb5d76242b5),
    ("Negative_Disp_Range", 48, 36, 0, 178, 0x1d8e1d22713fcee9, 0x77f3c5cdbc782a05, 0x8ec5011cb7fb425, 0x3563e2187fb4a965),
]


@pytest.mark.parametrize("row", GOLDEN_TABLE, ids=[r[0] for r in GOLDEN_TABLE])
def test_contract_fingerprints(row, O):
    tag, w, h, inv, rel, dh, ch, ih, rh = row
    if tag.startswith("Negative"):
        img = pattern(48, 36, 1, "noise")
        cfg = O.config(O.BALANCED, 8, -4)
    else:
        mode = {"Fast": O.FAST, "Balanced": O.BALANCED, "HighQuality": O.HIGH_QUALITY}[tag.split("_")[2]]
        img = pattern(33, 27, 1, "checker") if tag.startswith("Odd") else pattern(32, 24, 3, "noise")
        cfg = O.config(mode, 16, num_threads=1)
    out = O.pipeline(cfg, img, img)
    assert out["status"] == 0
    assert out["disparity"].shape == (h, w)
    assert int((out["disparity"] < 0).sum()) == inv
    assert int(out["reliable_mask"].sum()) == rel
    assert O.fnv1a64(out["disparity"]) == dh
    assert O.fnv1a64(out["confidence"]) == ch
    assert O.fnv1a64(out["invalid_reason"]) == ih
    assert O.fnv1a64(out["reliable_mask"]) == rh


def test_sgm_1d_known_answer(O):
    """tests/test_synthetic.cpp:26-71: 5x1x3 volume, P1=25, P2=80, horizontal path -> d(2) = 0."""
    w, h, D = 5, 1, 3
    cfg = O.config(O.BALANCED, D, P1=25, P2_base=80, adaptive_penalties=0)
    vol = np.zeros((h, w, D), np.uint16)
    for x in range(w):
        vol[0, x] = (30, 20, 70) if x == 2 else (10, 60, 70)
    acc = np.zeros((h, w, D), np.uint32)
    gray = np.full((h, w), 128, np.uint8)
    O.sgm_path(cfg, gray, vol, acc, 1, 0)
    rmin = np.zeros((h, w), np.int16)
    rmax = np.full((h, w), D, np.int16)
    disp, best, second = O.wta(cfg, acc, rmin, rmax)
    assert abs(float(disp[0, 2]) - 0.0) <= 0.01
    # path values of the reference's SgmOptimizer::aggregate_path for this volume (obtained by
    # running the reference build; they also follow by hand from the recurrence)
    assert acc[0].tolist() == [[10, 60, 70], [10, 85, 130], [30, 45, 150], [10, 75, 110], [10, 85, 150]]


FIX = Path(__file__).resolve().parent / "golden" / "reference_fixtures.npz"


def _fixture_cases():
    if not FIX.exists():
        return []
    with np.load(FIX) as z:
        return [str(c) for c in z["cases"]]


@pytest.mark.parametrize("case", _fixture_cases())
def test_oracle_matches_reference_fixtures(case, O):
    z = np.load(FIX)
    cfg = O.config_from_record(z[f"{case}/config"].tobytes())
    L, R = z[f"{case}/left"], z[f"{case}/right"]
    out = O.pipeline(cfg, L, R, stages=True)
    assert out["status"] == 0
    pairs = [("disparity", "disparity"), ("confidence", "confidence"), ("invalid_reason", "invalid_reason"),
             ("reliable_mask", "reliable_mask"), ("disp_wta", "disp_wta"), ("best", "best"), ("second", "second"),
             ("disp_right", "disp_right"), ("disp_refined", "disp_refined"), ("disp_lr", "disp_lr"),
             ("disp_fill", "disp_fill"), ("range_min", "range_min"), ("range_max", "range_max"),
             ("d_prior", "d_prior")]
    for mine, ref in pairs:
        assert same_bits(out[mine], z[f"{case}/{ref}"]), f"{case}: {mine}"
    assert out["support_count"] == int(z[f"{case}/support_count"])
    if f"{case}/cost_raw" in z.files:
        assert same_bits(out["cost_raw"], z[f"{case}/cost_raw"])
        assert same_bits(out["cost_agg"], z[f"{case}/cost_agg"])
        assert same_bits(out["sgm_sum"], z[f"{case}/sgm_sum"])


LIVE = [
    ("balanced_97x61_d24", 1, 24, 0, {}),
    ("fast_96x64_d32", 0, 32, 0, {}),
    ("hq_128x96_d32", 2, 32, 0, {}),
    ("balanced_min8", 1, 40, 8, {}),
    ("balanced_continuous_p2", 1, 24, 0, {"piecewise_p2": 0}),
    ("balanced_agg2", 1, 24, 0, {"agg_iterations": 2}),
]


@pytest.mark.parametrize("case", LIVE, ids=[c[0] for c in LIVE])
def test_oracle_matches_live_reference(case, O):
    if not O.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    name, mode, dmax, dmin, over = case
    w, h = {"balanced_97x61_d24": (97, 61)}.get(name, (128, 96) if "hq" in name else (96, 64))
    L, R = synth(w, h, dmax, cells=5, lo=max(0, dmin), hi=dmax * 3 // 4, patch=0.2 if mode == 2 else 0.0)
    cfg = O.config(mode, dmax, dmin, **over)
    o = O.pipeline(cfg, L, R, stages=True)
    r = O.ref_dump(cfg, L, R)
    assert r["status"] == 0
    for k in ("cost_raw", "cost_agg", "sgm_sum", "disp_wta", "best", "second", "disp_right", "range_min",
              "range_max", "d_prior", "disp_refined", "disp_lr", "disp_fill", "disparity", "confidence",
              "invalid_reason", "reliable_mask"):
        assert same_bits(o[k], r[k]), f"{name}: {k}"
