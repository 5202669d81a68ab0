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
