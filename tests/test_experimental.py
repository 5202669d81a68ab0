"""Experimental sub-pixel and inpaint variants (src/subpixel_estimator.cpp:58-119,
src/postprocess.cpp:170-239) behind their scopes: the oracle's restatement against the reference
(no GPU), stage by stage.

Every sub-pixel method (Legacy, CurvGate, ConfGate, Stabilized; default and explicit parameters)
and both inpaint methods (Legacy, ShadowReclass; default gap and an explicit one) run through the
reference's own scopes (ref_set_experimental) and the oracle's; the WTA map, the right-image map,
the filled map and the final outputs must match bit for bit.  The scope semantics of the Python
binding (nesting, restore on exit, thread-local) are checked without a GPU.
"""
import threading

import numpy as np
import pytest

from helpers import same_bits, synth

SCOPES = [
    # (sp_method, sp_param, ip_method, ip_gap)
    (1, 0.0, 0, 32), (1, 12.0, 0, 32), (2, 0.0, 0, 32), (2, 0.3, 0, 32), (3, 0.0, 0, 32), (3, 1.5, 0, 32),
    (0, 0.0, 1, 32), (0, 0.0, 1, 8), (0, 0.0, 0, 5), (3, 2.0, 1, 48),
]
CONFIGS = [
    # mode, w, h, dmax, dmin, patch
    (1, 96, 64, 32, 0, 0.25),
    (0, 80, 48, 24, 0, 0.3),
    (2, 96, 72, 32, 0, 0.3),
]


@pytest.fixture
def scoped(O):
    yield
    O.set_experimental()
    if O.ref_available():
        O.set_experimental(reference=True)


@pytest.mark.parametrize("scope", SCOPES, ids=[f"sp{a}_{b}_ip{c}_{d}" for a, b, c, d in SCOPES])
def test_oracle_matches_reference_under_scopes(scope, O, scoped):
    if not O.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    for mode, w, h, dmax, dmin, patch in CONFIGS:
        cfg = O.config(mode, dmax, dmin)
        L, R = synth(w, h, dmax, patch=patch, seed=w + h + mode)
        O.set_experimental(*scope)
        O.set_experimental(*scope, reference=True)
        got = O.pipeline(cfg, L, R, stages=True)
        ref = O.ref_dump(cfg, L, R)
        assert ref["status"] == 0 and got["status"] == 0
        for k in ("disp_wta", "disp_right", "disp_lr", "disp_fill", "disparity", "confidence", "invalid_reason",
                  "reliable_mask"):
            assert same_bits(got[k], ref[k]), (scope, mode, k)


def test_scopes_change_something(O, scoped):
    """Each variant moves some pixels (the cases above are not vacuous)."""
    cfg = O.config(1, 32)
    L, R = synth(96, 64, 32, patch=0.25, seed=7)
    base = O.pipeline(cfg, L, R, stages=True)
    for scope in [(1, 0.0, 0, 32), (2, 0.0, 0, 32), (3, 0.0, 0, 32), (0, 0.0, 1, 32), (0, 0.0, 0, 5)]:
        O.set_experimental(*scope)
        v = O.pipeline(cfg, L, R, stages=True)
        assert not same_bits(v["disparity"], base["disparity"]), scope
    O.set_experimental()


def test_python_scopes_nest_and_are_thread_local(apg):
    assert apg._get_experimental() == (0, 0.0, 0, 32)
    with apg.ExperimentalSubpixelScope("stabilized", 2.5):
        with apg.ExperimentalInpaintScope(apg.InpaintMethod.ShadowReclass, 16):
            assert apg._get_experimental() == (3, 2.5, 1, 16)
            seen = []
            t = threading.Thread(target=lambda: seen.append(apg._get_experimental()))
            t.start()
            t.join()
            assert seen == [(0, 0.0, 0, 32)]
        assert apg._get_experimental() == (3, 2.5, 0, 32)
    assert apg._get_experimental() == (0, 0.0, 0, 32)
    with pytest.raises(ValueError):
        apg.ExperimentalInpaintScope("bogus")
    with apg.ExperimentalSubpixelScope("legacy", collect_telemetry=True):
        with apg.ExperimentalInpaintScope("legacy", collect_telemetry=True):
            assert apg._get_telemetry_flags() == (1, 1)
        assert apg._get_telemetry_flags() == (1, 0)
        assert apg.ExperimentalSubpixelScope.current_telemetry().candidate_pixels == 0
    assert apg._get_telemetry_flags() == (0, 0)


TEL_CASES = [(1, (2, 0.0, 1, 16), 0), (2, (3, 0.0, 0, 32), 0), (1, (0, 0.0, 0, 32), 1), (0, (1, 6.0, 0, 8), 0)]


@pytest.mark.parametrize("case", TEL_CASES, ids=[f"m{m}_sp{s[0]}_ip{s[2]}_h{h}" for m, s, h in TEL_CASES])
def test_telemetry_oracle_matches_reference(case, O, scoped):
    """SubpixelTelemetry / InpaintTelemetry of one frame (the reference's own scopes with
    collect_telemetry, through its StereoSession) against the oracle's, the hierarchical coarse
    pass included."""
    if not O.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    mode, scope, hier = case
    L, R = synth(96, 64, 32, patch=0.25, seed=21 + mode)
    O.set_experimental(*scope, sp_telemetry=True, ip_telemetry=True)
    O.set_experimental(*scope, reference=True, sp_telemetry=True, ip_telemetry=True)
    O.pipeline(O.config(mode, 32, hier_enable=hier), L, R)
    s = O.RefSession(O.config(mode, 32, volume_backend=2, hier_enable=hier), bounded_reuse=True)
    assert s.process(L, R)["status"] == 0
    (sa, ia), (sb, ib) = O.get_telemetry(), O.get_telemetry(reference=True)
    assert sa.pop("sum_abs_delta") == pytest.approx(sb.pop("sum_abs_delta"), rel=1e-12)
    assert sa == sb and ia == ib
    assert sa["candidate_pixels"] > 0 and ia["total_invalid_pixels"] > 0
