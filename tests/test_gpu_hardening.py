"""Session semantics of the reference's tests/test_hardening.cpp, through the C ABI (backend 3).

That file drives the reference's C++ StereoMatcher / StereoSession, which this library does not
ship; the same cases run here through apg_session_* with a device present: the pre-compute budget
gate leaves 0 bytes allocated (:41-62), a failed frame neither counts nor poisons the session
(:64-91), BoundedReuse allocates once and then reuses (:93-131), retained capacity is reported
after a large-to-small switch (:133-168), and ReleasePerFrame keeps 0 bytes between frames.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OK, EMPTY_INPUT, SIZE_MISMATCH, RESOURCE_LIMIT = 0, 1, 2, 6


def _session(L, mode=0, policy=0, budget=0, dmax=32):
    from apg_sgm_b200 import _lib
    o = _lib.SessionOptions()
    o.struct_size = C.sizeof(_lib.SessionOptions)
    o.quality_mode, o.memory_policy, o.max_retained_bytes = mode, policy, budget
    o.min_disparity, o.max_disparity, o.backend = 0, dmax, 3
    s = L.apg_session_create_ex(C.byref(o))
    assert s
    return s


def _view(a, stride=None):
    from apg_sgm_b200 import _lib
    h, w = a.shape[:2]
    return C.byref(_lib.ImageView(a.ctypes.data, w, h, stride if stride is not None else a.strides[0], 1))


def _counters(L, s):
    ms = (C.c_double * 11)()
    cnt = (C.c_size_t * 4)()
    assert L.apgcu_session_get_stats(s, ms, cnt) == OK
    return [int(v) for v in cnt]  # allocation, reuse, peak, retained


def _disparity(L, r):
    p = L.apg_result_get_disparity(r, None, None)
    assert p
    return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_float)), shape=(48 * 64,))


def _lib_handle(apg):
    from apg_sgm_b200 import _lib
    return _lib.lib()


def test_budget_gate_allocates_nothing(apg):
    L = _lib_handle(apg)
    s = _session(L, mode=0, budget=10 * 1024, dmax=64)
    r = L.apg_result_create()
    img = np.full((240, 320), 128, np.uint8)
    assert L.apg_session_process(s, _view(img), _view(img), r) == RESOURCE_LIMIT
    assert L.apg_session_get_allocated_bytes(s) == 0
    assert L.apg_session_get_frame_count(s) == 0
    L.apg_result_destroy(r)
    L.apg_session_destroy(s)


def test_invalid_stride_is_size_mismatch(apg):
    L = _lib_handle(apg)
    s = _session(L)
    r = L.apg_result_create()
    buf = np.zeros(24 * 32, np.uint8)
    v = _view(buf.reshape(24, 32), stride=16)
    assert L.apg_session_process(s, v, v, r) == SIZE_MISMATCH
    assert L.apg_session_get_allocated_bytes(s) == 0
    L.apg_result_destroy(r)
    L.apg_session_destroy(s)


@pytest.mark.parametrize("policy", [0, 1])
def test_fault_recovery_across_frames(apg, policy):
    L = _lib_handle(apg)
    s = _session(L, mode=1, policy=policy)
    r = L.apg_result_create()
    img = np.full((48, 64), 100, np.uint8)
    assert L.apg_session_process(s, _view(img), _view(img), r) == OK
    assert L.apg_session_get_frame_count(s) == 1
    first = _disparity(L, r).copy()
    assert L.apg_session_process(s, None, _view(img), r) == EMPTY_INPUT
    assert L.apg_session_get_frame_count(s) == 1
    assert L.apg_session_get_last_error(s)
    assert L.apg_session_process(s, _view(img), _view(img), r) == OK
    assert L.apg_session_get_frame_count(s) == 2
    w, h = C.c_int(), C.c_int()
    p = L.apg_result_get_disparity(r, C.byref(w), C.byref(h))
    assert p and (w.value, h.value) == (64, 48)
    again = _disparity(L, r)
    assert np.array_equal(first.view(np.uint32), again.view(np.uint32))
    L.apg_result_destroy(r)
    L.apg_session_destroy(s)


def test_bounded_reuse_steady_state(apg):
    L = _lib_handle(apg)
    s = _session(L, mode=0, policy=1, dmax=32)
    r = L.apg_result_create()
    img = np.full((48, 64), 150, np.uint8)
    for frame in range(3):
        assert L.apg_session_process(s, _view(img), _view(img), r) == OK
        alloc, reuse, _, retained = _counters(L, s)
        assert (alloc, reuse) == (1, frame)
        assert retained == L.apg_session_get_allocated_bytes(s) > 0
    L.apg_result_destroy(r)
    L.apg_session_destroy(s)


def test_retained_capacity_large_to_small(apg):
    L = _lib_handle(apg)
    s = _session(L, mode=0, policy=1, dmax=32)
    r = L.apg_result_create()
    large = np.full((96, 128), 120, np.uint8)
    small = np.full((48, 64), 120, np.uint8)
    assert L.apg_session_process(s, _view(large), _view(large), r) == OK
    large_bytes = L.apg_session_get_allocated_bytes(s)
    assert large_bytes > 0 and _counters(L, s)[3] == large_bytes
    assert L.apg_session_process(s, _view(small), _view(small), r) == OK
    small_bytes = L.apg_session_get_allocated_bytes(s)
    assert _counters(L, s)[3] == small_bytes
    assert small_bytes >= large_bytes
    L.apg_result_destroy(r)
    L.apg_session_destroy(s)


def test_release_per_frame_keeps_nothing(apg):
    L = _lib_handle(apg)
    s = _session(L, mode=1, policy=0, dmax=32)
    r = L.apg_result_create()
    img = np.full((48, 64), 90, np.uint8)
    for _ in range(2):
        assert L.apg_session_process(s, _view(img), _view(img), r) == OK
        assert L.apg_session_get_allocated_bytes(s) == 0
    alloc, reuse, peak, _ = _counters(L, s)
    assert (alloc, reuse) == (2, 0) and peak > 0
    L.apg_result_destroy(r)
    L.apg_session_destroy(s)


INTERNAL_ERROR = 8


@pytest.mark.parametrize("policy", [0, 1])
def test_refiner_wait_runs_out_then_session_recovers(apg, O, policy):
    """A bounded device wait that runs out (the fault-recovery case of test_hardening.cpp:64-91,
    made on the device without faulting it).  With the refiner's poll budget at one poll, a band
    stops waiting for the band above almost at once: the kernel sets the frame's error word, every
    band returns, and apg_session_process reports INTERNAL_ERROR with a last_error, counting no
    frame.  The next frame on the same session, with the default budget, is bit-exact with the
    oracle.  160x128 HighQuality has four refiner bands per pass, three of which wait."""
    from helpers import synth, to_oracle
    L = _lib_handle(apg)
    cfg = apg.config_from_mode(2, 32)
    s = L.apgcu_session_create_config(C.byref(cfg), policy, 0)
    assert s
    r = L.apg_result_create()
    left, right = synth(160, 128, 32, patch=0.2, seed=9)
    assert L.apgcu_session_set_tuning(s, b"refine_spin_limit", 1) == OK
    assert L.apgcu_session_set_tuning(s, b"refine_spin_limit", -1) == 4  # INVALID_CONFIG
    assert L.apgcu_session_set_tuning(s, b"no_such_key", 1) == 4
    rc = L.apg_session_process(s, _view(left), _view(right), r)
    assert rc == INTERNAL_ERROR, rc
    assert b"wavefront wait timed out" in L.apg_session_get_last_error(s)
    assert L.apg_session_get_frame_count(s) == 0
    assert not L.apg_result_get_disparity(r, None, None)
    assert L.apgcu_session_set_tuning(s, b"refine_spin_limit", 0) == OK
    assert L.apg_session_process(s, _view(left), _view(right), r) == OK
    assert L.apg_session_get_frame_count(s) == 1
    assert L.apg_session_get_last_error(s) == b""
    want = O.pipeline(to_oracle(O, cfg), left, right)
    w, h = C.c_int(), C.c_int()
    p = L.apg_result_get_disparity(r, C.byref(w), C.byref(h))
    got = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_float)), shape=(128, 160)).copy()
    assert np.array_equal(got.view(np.uint32), want["disparity"].view(np.uint32))
    L.apg_result_destroy(r)
    L.apg_session_destroy(s)


def test_engine_refiner_wait_runs_out(apg, O):
    """The same through the engine entry point: the failed frame raises with the engine's error,
    the next one (default budget) equals the oracle."""
    from helpers import same_bits, synth, to_oracle
    cfg = apg.config_from_mode(2, 32)
    left, right = synth(160, 128, 32, patch=0.2, seed=10)
    eng = apg.Engine(cfg)
    eng.set_tuning("refine_spin_limit", 1)
    with pytest.raises(RuntimeError, match="wavefront wait timed out"):
        eng.process(left, right)
    eng.set_tuning("refine_spin_limit", 0)
    got = eng.process(left, right)
    want = O.pipeline(to_oracle(O, cfg), left, right)
    for k in ("disparity", "confidence", "invalid_reason", "reliable_mask"):
        assert same_bits(got[k], want[k]), k
    eng.close()
