"""Accuracy metrics on the GPU (apgcu_evaluate_stereo) against the oracle and the reference.

Every case of tests/test_metrics.py runs through the device path with host buffers and with
CUDA-tensor buffers; the record must equal the oracle's (and the reference's frozen fixtures)
field for field.  Tolerance: counts and count ratios are exact; the means formed from double sums
of float errors are exact whenever the reference's sequential double sum is exact (all
`quantised` cases); on the one unquantised case they may differ from the reference's by one
float ulp, because the device adds the same errors in another order.  At 1920 x 1080 the
engine's own output is scored against the synthetic ground truth and checked against the oracle.
"""
from pathlib import Path

import numpy as np
import pytest

from helpers import metric_case, same_metrics
from test_metrics import CASES, _oracle, run_case

pytestmark = pytest.mark.gpu

FIX = Path(__file__).resolve().parent / "golden" / "metrics_fixtures.npz"
SUM_FIELDS = {"epe", "edge_epe", "nonedge_epe", "refine_epe_delta", "post_epe_delta", "total_epe_delta"} | {
    f"reg_{r}.epe" for r in ("all", "noc", "occ", "boundary", "non_boundary", "low_texture", "high_texture")}


def _gpu(apg):
    return lambda est, gt, rng, b, a, vis, mx, left, thr: apg.evaluate_stereo(est, gt, rng, b, a, vis, mx, left, thr)


def _check(bad, quantised):
    if quantised:
        assert not bad, bad
        return
    for k, va, vb in bad:
        assert k in SUM_FIELDS, (k, va, vb)
        assert abs(np.float32(va) - np.float32(vb)) <= np.spacing(np.float32(max(abs(va), abs(vb)))), (k, va, vb)


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_gpu_metrics_match_oracle(case, O, apg):
    got = run_case(_gpu(apg), case)
    want = run_case(_oracle(O), case)
    _check(same_metrics(got, want), case[5])
    if FIX.exists():
        z = np.load(FIX)
        if f"{case[0]}/record" in z:
            ref = O.StereoMetricsRec.from_buffer_copy(z[f"{case[0]}/record"].tobytes())
            _check(same_metrics(got, ref), case[5])


def test_gpu_metrics_device_buffers(apg):
    import torch
    d = metric_case(257, 131, 11, 3)
    host = apg.evaluate_stereo(d["est"], d["gt"], d["range"], d["before"], d["after"], d["vis"], 1e5, d["left"])
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in d.items() if k != "range"}
    rng = tuple(torch.from_numpy(v).cuda() for v in d["range"])
    dev = apg.evaluate_stereo(t["est"], t["gt"], rng, t["before"], t["after"], t["vis"], 1e5, t["left"])
    assert not same_metrics(host, dev)
    with pytest.raises(ValueError):
        apg.evaluate_stereo(t["est"], d["gt"])


def test_gpu_metrics_empty_and_errors(apg):
    z = np.zeros((0, 5), np.float32)
    m = apg.evaluate_stereo(z, z)
    assert m.total_pixels == 0 and m.evaluated_pixels == 0
    with pytest.raises(ValueError):
        apg.evaluate_stereo(np.zeros((4, 5), np.float32), np.zeros((4, 6), np.float32))


def test_gpu_metrics_1080p_engine_output(O, apg):
    """Score a Balanced 1920x1080 D256 engine output against its synthetic ground truth, with the
    frame's ranges, the WTA / refined maps of an HQ run and the left image; equal to the oracle."""
    from apg_sgm_b200 import synthetic as S
    spec = S.PairSpec(1920, 1080, 256, 16, 0, 240, 0.2)
    L, R, gt = S.make_pair(spec, 7)
    gt = (np.round(gt.astype(np.float64) * 256) / 256).astype(np.float32)
    e = apg.Engine(apg.config_from_mode(2, 256))
    out = e.process(L, R)
    rmin, rmax = e.dump("range_min"), e.dump("range_max")
    before, after = e.dump("disp_wta"), e.dump("disp_refined")
    e.close()
    est = out["disparity"]
    vis = np.where(np.arange(1920)[None, :] - np.round(gt) >= 0, 255, 0).astype(np.uint8)
    got = apg.evaluate_stereo(est, gt, (rmin, rmax), before, after, vis, 1e5, L)
    want = O.evaluate_stereo(est, gt, (rmin, rmax), before, after, vis, 1e5, L)
    bad = same_metrics(got, want)
    # engine disparities carry arbitrary sub-pixel fractions: only the double-sum means may differ
    _check(bad, False)
    assert got.evaluated_pixels == 1920 * 1080 and got.has_refine_stats and got.has_range
    # a scored map, not a quality target (the synthetic pair has 20% flat patches)
    assert got.valid_pixels > 0 and 0.0 < got.epe < 64.0
    assert got.reg_all.total_pixels == got.evaluated_pixels


@pytest.mark.parametrize("w,h,dmax,max_sup", [(320, 240, 64, 4000), (240, 160, 48, 60), (200, 120, 64, 200)])
def test_engine_supports_and_support_metrics(O, apg, w, h, dmax, max_sup):
    """The prior's support list (Engine.supports) equals the oracle's extract_supports in order and
    value -- the stratified budget (max 4000) and the uniform sampling (60 < non-empty cells) -- and
    evaluate_supports on the GPU equals the oracle's on it."""
    from helpers import synth, to_oracle
    cfg = apg.config_from_mode(2, dmax, prior_max_supports=max_sup)
    L, R = synth(w, h, dmax, patch=0.2, seed=w + max_sup)
    e = apg.Engine(cfg)
    e.process(L, R)
    sx, sy, sd, sc = e.supports()
    e.close()
    ox, oy, od, oc = O.supports(to_oracle(O, cfg), L, R)
    assert len(sx) == len(ox) > 0
    assert np.array_equal(sx, ox) and np.array_equal(sy, oy)
    assert np.array_equal(sd.view(np.uint32), od.view(np.uint32)) and np.array_equal(sc.view(np.uint32), oc.view(np.uint32))
    d = metric_case(w, h, 5)
    for vis in (None, d["vis"]):
        got = apg.evaluate_supports((sx, sy, sd), d["gt"], vis)
        want = O.evaluate_supports(sx, sy, sd, d["gt"], vis)
        assert got.to_dict() == want.to_dict()
