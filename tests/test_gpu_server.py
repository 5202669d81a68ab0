"""Served form (apgcu_server_*): each result is the same alone and in the mix.

A burst of requests of four sizes and three quality modes, in shuffled order, is served with
several slots (their work overlaps on the device); every output must equal, bit for bit, the
single-pair engine's output for that pair.  A small HBM budget forces engine evictions without
changing any result, and a request larger than the whole budget is refused.
"""
import numpy as np
import pytest

from helpers import same_bits, synth

pytestmark = pytest.mark.gpu

KEYS = ("disparity", "confidence", "invalid_reason", "reliable_mask")
SIZES = [(160, 96, 64), (200, 120, 128), (256, 64, 192), (192, 108, 256)]


def _pool():
    pool = []
    for i, (w, h, dmax) in enumerate(SIZES):
        for mode in (1, 0, 2):
            L, R = synth(w, h, dmax, cells=5, lo=0, hi=dmax - 8, patch=0.2 if mode == 2 else 0.0, seed=60 + i)
            pool.append((mode, dmax, L, R))
    return pool


def _alone(apg, pool):
    want = []
    for mode, dmax, L, R in pool:
        e = apg.Engine(apg.config_from_mode(mode, dmax))
        want.append(e.process(L, R))
        e.close()
    return want


def _serve(apg, pool, order, **kw):
    srv = apg.Server(**kw)
    tickets = [(i, srv.submit(pool[i][2], pool[i][3], mode=pool[i][0], max_disparity=pool[i][1])) for i in order]
    got = []
    for i, t in tickets:
        o, lat = srv.wait(t)
        assert lat > 0
        got.append((i, o))
    st = srv.stats()
    srv.close()
    return got, st


def test_served_results_equal_alone(apg):
    pool = _pool()
    want = _alone(apg, pool)
    order = np.random.default_rng(7).permutation(np.repeat(np.arange(len(pool)), 3))
    got, st = _serve(apg, pool, order, slots=4)
    for i, o in got:
        for k in KEYS:
            assert same_bits(o[k], want[i][k]), (i, k)
    assert st["completed"] == len(order) and st["failed"] == 0
    assert st["peak_in_flight"] >= 2


def test_served_small_budget_evicts_and_matches(apg):
    pool = _pool()
    want = _alone(apg, pool)
    biggest = max(apg.workspace_bytes(apg.config_from_mode(m, d), L.shape[1], L.shape[0]) for m, d, L, _ in pool)
    order = np.random.default_rng(8).permutation(np.repeat(np.arange(len(pool)), 2))
    got, st = _serve(apg, pool, order, slots=3, hbm_budget_gb=1.5 * biggest / (1 << 30))
    for i, o in got:
        for k in KEYS:
            assert same_bits(o[k], want[i][k]), (i, k)
    assert st["evictions"] > 0
    assert st["peak_reserved_bytes"] <= st["budget_bytes"]


def test_served_request_beyond_budget_is_refused(apg):
    L, R = synth(320, 240, 128)
    srv = apg.Server(slots=1, hbm_budget_gb=1e-3)
    t = srv.submit(L, R, mode=1, max_disparity=128)
    with pytest.raises(RuntimeError, match=r"\[6\].*budget"):
        srv.wait(t)
    srv.close()


def test_served_warm_pool_matches(apg):
    """Engines created ahead by reserve() (warmed on a blank pair) give the same results, and the
    requests that find them allocate nothing more."""
    pool = _pool()
    want = _alone(apg, pool)
    srv = apg.Server(slots=2)
    for mode, dmax, L, _ in pool:
        srv.reserve(L.shape[1], L.shape[0], mode=mode, max_disparity=dmax, count=2)
    reserved = srv.stats()["reserved_bytes"]
    order = np.random.default_rng(9).permutation(np.repeat(np.arange(len(pool)), 2))
    tickets = [(i, srv.submit(pool[i][2], pool[i][3], mode=pool[i][0], max_disparity=pool[i][1])) for i in order]
    for i, t in tickets:
        o, _ = srv.wait(t)
        for k in KEYS:
            assert same_bits(o[k], want[i][k]), (i, k)
    st = srv.stats()
    assert st["reserved_bytes"] == reserved and st["evictions"] == 0
    srv.close()


def test_served_reserve_beyond_budget_is_refused(apg):
    srv = apg.Server(slots=1, hbm_budget_gb=1e-3)
    with pytest.raises(RuntimeError, match=r"\[6\]"):
        srv.reserve(320, 240, mode=1, max_disparity=128)
    srv.close()


def test_served_into_caller_buffers(apg):
    pool = _pool()[:3]
    want = _alone(apg, pool)
    srv = apg.Server(slots=2)
    outs = []
    for mode, dmax, L, R in pool:
        h, w = L.shape
        o = {"disparity": np.full((h, w), 7, np.float32), "confidence": np.full((h, w), 7, np.float32),
             "invalid_reason": np.full((h, w), 7, np.uint8), "reliable_mask": np.full((h, w), 7, np.uint8)}
        outs.append((o, srv.submit(L, R, mode=mode, max_disparity=dmax, out=o)))
    for i, (o, t) in enumerate(outs):
        got, _ = srv.wait(t)
        assert got is o
        for k in KEYS:
            assert same_bits(o[k], want[i][k]), (i, k)
    with pytest.raises(ValueError):
        srv.submit(pool[0][2], pool[0][3], out={k: np.zeros((1, 1), np.float32) for k in KEYS})
    srv.close()


def test_server_stop_completes_queued_requests(apg):
    """Destroying a server with requests still queued completes them with an error, so a thread
    waiting for one returns (no hang); the requests that ran are unaffected."""
    import ctypes as C
    import threading
    import time

    from apg_sgm_b200._lib import lib

    L, R = synth(1280, 720, 128, cells=6, lo=0, hi=120, patch=0.2, seed=81)
    srv = apg.Server(slots=1)
    tickets = [srv.submit(L, R, mode=2, max_disparity=128) for _ in range(48)]
    res = {}

    def waiter():
        lat = C.c_double()
        res["rc"] = lib().apgcu_server_wait(srv._h, tickets[-1], C.byref(lat))

    t = threading.Thread(target=waiter, daemon=True)
    t.start()
    time.sleep(0.05)
    srv.close()  # joins the worker after its current request; the rest complete with an error
    t.join(timeout=120)
    assert not t.is_alive(), "a thread waiting on a queued request did not return after the server stopped"
    assert res["rc"] in (0, 8), res
