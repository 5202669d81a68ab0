"""Experimental sub-pixel and inpaint variants on the GPU against the oracle, under the same scopes.

The engine reads the calling thread's scopes once per frame (WTA and right-image sub-pixel step,
hole fill method and gap); every stage it dumps must equal the oracle's under the same settings.
Also: the batched form run inside a scope, the column-tile cost kernel, the hierarchical mode's
coarse pass (which runs the same kernels on the same thread), and a worker thread that sees the
default scope.
"""
import threading

import numpy as np
import pytest

from helpers import same_bits, synth, to_oracle

pytestmark = pytest.mark.gpu

SCOPES = [(1, 0.0, 0, 32), (1, 12.0, 0, 32), (2, 0.0, 0, 32), (2, 0.3, 0, 32), (3, 0.0, 0, 32), (3, 1.5, 0, 32),
          (0, 0.0, 1, 32), (0, 0.0, 1, 8), (0, 0.0, 0, 5), (3, 2.0, 1, 48)]
CONFIGS = [(1, 200, 96, 64, 0, 0.25), (0, 160, 80, 64, 0, 0.3), (2, 160, 96, 64, 0, 0.3), (1, 128, 64, 40, -16, 0.2)]
STAGES = ("disp_wta", "disp_right", "disp_lr", "disp_fill")
MAPS = ("disparity", "confidence", "invalid_reason", "reliable_mask")


def _scope(apg, s):
    sm, sp, im, ig = s

    class Both:
        def __enter__(self):
            self.a = apg.ExperimentalSubpixelScope(sm, sp)
            self.b = apg.ExperimentalInpaintScope(im, ig)
            self.a.__enter__()
            self.b.__enter__()

        def __exit__(self, *e):
            self.b.__exit__(*e)
            self.a.__exit__(*e)

    return Both()


@pytest.fixture
def oracle_scope(O):
    yield
    O.set_experimental()


@pytest.mark.parametrize("scope", SCOPES, ids=[f"sp{a}_{b}_ip{c}_{d}" for a, b, c, d in SCOPES])
def test_engine_matches_oracle_under_scopes(scope, O, apg, oracle_scope):
    for mode, w, h, dmax, dmin, patch in CONFIGS:
        cfg = apg.config_from_mode(mode, dmax, dmin)
        L, R = synth(w, h, dmax, patch=patch, seed=w + h + mode)
        e = apg.Engine(cfg, debug=apg.DEBUG_RAW_COST)
        with _scope(apg, scope):
            out = e.process(L, R)
        dumps = {k: e.dump(k) for k in STAGES}
        e.close()
        O.set_experimental(*scope)
        ref = O.pipeline(to_oracle(O, cfg), L, R, stages=True)
        for k in STAGES:
            assert same_bits(dumps[k], ref[k]), (scope, mode, k)
        for k in MAPS:
            assert same_bits(out[k], ref[k]), (scope, mode, k)


def test_tile_cost_kernel_and_hierarchical_under_scope(O, apg, oracle_scope):
    scope = (3, 1.5, 1, 16)
    L, R = synth(200, 96, 64, patch=0.25, seed=77)
    O.set_experimental(*scope)
    cfg = apg.config_from_mode(1, 64)
    e = apg.Engine(cfg)
    e.set_tuning("cost_kernel", 1)
    with _scope(apg, scope):
        out = e.process(L, R)
    e.close()
    ref = O.pipeline(to_oracle(O, cfg), L, R)
    for k in MAPS:
        assert same_bits(out[k], ref[k]), k
    hcfg = apg.config_from_mode(1, 64, hier_enable=1)
    e = apg.Engine(hcfg)
    with _scope(apg, scope):
        out = e.process(L, R)
    e.close()
    ref = O.pipeline(to_oracle(O, hcfg), L, R)
    for k in MAPS:
        assert same_bits(out[k], ref[k]), ("hier", k)


def test_batch_under_scope_and_default_elsewhere(O, apg, oracle_scope):
    scope = (2, 0.2, 1, 32)
    sizes = [(160, 96, 64), (200, 120, 64), (160, 96, 64)]
    pairs = [synth(w, h, d, patch=0.25, seed=90 + i) for i, (w, h, d) in enumerate(sizes)]
    b = apg.Batch(apg.config_from_mode(1, 64))
    with _scope(apg, scope):
        got = b.process([(L, R, d) for (L, R), (_, _, d) in zip(pairs, sizes)])
    plain = b.process([(L, R, d) for (L, R), (_, _, d) in zip(pairs, sizes)])  # outside the scope again
    b.close()
    cfg = apg.config_from_mode(1, 64)
    for i, (L, R) in enumerate(pairs):
        O.set_experimental(*scope)
        want = O.pipeline(to_oracle(O, cfg), L, R)
        O.set_experimental()
        base = O.pipeline(to_oracle(O, cfg), L, R)
        for k in MAPS:
            assert same_bits(got[i][k], want[k]), (i, k)
            assert same_bits(plain[i][k], base[k]), (i, k)
    # a thread of its own sees the default scope while this one holds another
    L, R = pairs[0]
    base = O.pipeline(to_oracle(O, cfg), L, R)
    res = {}

    def worker():
        e = apg.Engine(cfg)
        res["out"] = e.process(L, R)
        e.close()

    with _scope(apg, scope):
        t = threading.Thread(target=worker)
        t.start()
        t.join()
    for k in MAPS:
        assert same_bits(res["out"][k], base[k]), k


TEL_CASES = [(1, (2, 0.0, 1, 16), 0), (2, (3, 0.0, 0, 32), 0), (1, (0, 0.0, 0, 32), 1), (0, (1, 6.0, 0, 8), 0)]


@pytest.mark.parametrize("case", TEL_CASES, ids=[f"m{m}_sp{s[0]}_ip{s[2]}_h{h}" for m, s, h in TEL_CASES])
def test_telemetry_matches_oracle(case, O, apg, oracle_scope):
    """The scopes' telemetry counted on the device (WTA sub-pixel step, hole fill, run lengths; the
    hierarchical coarse pass included) equals the oracle's; two frames accumulate; the batched form
    collects its pairs'."""
    mode, (sm, sp, im, ig), hier = case
    L, R = synth(160, 96, 48, patch=0.25, seed=31 + mode)
    cfg = apg.config_from_mode(mode, 48, hier_enable=hier)
    O.set_experimental(sm, sp, im, ig, sp_telemetry=True, ip_telemetry=True)
    O.pipeline(to_oracle(O, cfg), L, R)
    O.pipeline(to_oracle(O, cfg), L, R)
    want_sp, want_ip = O.get_telemetry()
    e = apg.Engine(cfg)
    with apg.ExperimentalSubpixelScope(sm, sp, collect_telemetry=True), \
            apg.ExperimentalInpaintScope(im, ig, collect_telemetry=True):
        e.process(L, R)
        e.process(L, R)
        got_sp = apg.ExperimentalSubpixelScope.current_telemetry()
        got_ip = apg.ExperimentalInpaintScope.current_telemetry()
    e.close()
    for k, v in want_sp.items():
        if k == "sum_abs_delta":
            assert got_sp.sum_abs_delta == pytest.approx(v, rel=1e-12)
        else:
            assert getattr(got_sp, k) == v, k
    for k, v in want_ip.items():
        assert getattr(got_ip, k) == v, k
    assert got_sp.candidate_pixels > 0 and got_ip.total_invalid_pixels > 0
    assert 0.0 <= got_sp.applied_ratio() <= 1.0 and 0.0 <= got_ip.fill_ratio() <= 1.0
    # the batched form, two pairs of this size: the same counters as two engine frames
    if not hier:
        b = apg.Batch(cfg)
        with apg.ExperimentalSubpixelScope(sm, sp, collect_telemetry=True), \
                apg.ExperimentalInpaintScope(im, ig, collect_telemetry=True):
            b.process([(L, R), (L, R)])
            bsp = apg.ExperimentalSubpixelScope.current_telemetry()
            bip = apg.ExperimentalInpaintScope.current_telemetry()
        b.close()
        assert bsp.candidate_pixels == want_sp["candidate_pixels"] and bip.route_counts == want_ip["route_counts"]
