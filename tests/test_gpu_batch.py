"""Batched form (apgcu_batch_*): every pair's outputs equal the single-pair engine's, bit for bit.

Covers pairs of uneven sizes and disparity ranges in one call (several buckets, Dp 64 / 128 / 192),
a second call with new pairs (replay of the cached per-bucket graphs), each option (graphs off,
per-pair SGM instead of the persistent batched one, half-warp chains, a capped persistent grid),
Fast and HighQuality modes (the latter through the Path8 fold and the uncaptured refine), device
buffers, and the rejection of an invalid pair.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import same_bits, synth

pytestmark = pytest.mark.gpu

KEYS = ("disparity", "confidence", "invalid_reason", "reliable_mask")
# (w, h, dmax, count)
MIX = [(160, 96, 64, 3), (130, 70, 48, 2), (200, 120, 128, 2), (256, 64, 192, 1)]


def _pairs(seed0, mix=MIX, patch=0.0):
    out, s = [], seed0
    for w, h, dmax, cnt in mix:
        for _ in range(cnt):
            L, R = synth(w, h, dmax, cells=5, lo=0, hi=dmax - 4, patch=patch, seed=s)
            out.append((L, R, dmax))
            s += 1
    return out


def _single(apg, mode, pairs):
    res = []
    for L, R, dmax in pairs:
        eng = apg.Engine(apg.config_from_mode(mode, dmax))
        res.append(eng.process(L, R))
        eng.close()
    return res


def _check(got, want):
    assert len(got) == len(want)
    for i, (g, w) in enumerate(zip(got, want)):
        for k in KEYS:
            assert same_bits(g[k], w[k]), (i, k, int((g[k] != w[k]).sum()))


@pytest.mark.parametrize("mode", [1, 0])
def test_batch_equals_single_pairs_and_replays(apg, mode):
    b = apg.Batch(apg.config_from_mode(mode, 128))
    for seed in (100, 200):  # the second call replays the graphs captured by the first
        pairs = _pairs(seed)
        _check(b.process(pairs), _single(apg, mode, pairs))
    b.close()


@pytest.mark.parametrize("opts", [{"graphs": 0}, {"batched_sgm": 0}, {"sgm_lanes": 16}, {"unified_sgm": 0},
                                  {"unified_sgm": 0, "graphs": 0},
                                  {"max_blocks_per_sm": 1, "autotune": 0}, {"cost_tile": 256}, {"cost_tile": 64}])
def test_batch_options_change_no_result(apg, opts):
    pairs = _pairs(300, mix=[(160, 96, 64, 2), (200, 120, 128, 2)])
    b = apg.Batch(apg.config_from_mode(1, 128), **opts)
    _check(b.process(pairs), _single(apg, 1, pairs))
    b.close()


@pytest.mark.parametrize("mode", [1, 0])
def test_batch_one_sgm_launch_over_all_ranges(apg, mode):
    """Pairs of every padded range (Dp 64, 128, 192, 256) and four sizes share one persistent SGM
    launch per phase; calls with another composition (a bucket missing, a bucket with more pairs)
    build their own plan and graph, and a repeated composition replays its graph."""
    mix = [(150, 80, 60, 2), (200, 100, 128, 1), (260, 60, 190, 2), (300, 50, 250, 1)]
    b = apg.Batch(apg.config_from_mode(mode, 128))
    comps = [(600, mix), (610, mix[1:]), (620, [(150, 80, 60, 3)] + mix[1:]), (630, mix)]
    for seed, m in comps:
        pairs = _pairs(seed, mix=m)
        _check(b.process(pairs), _single(apg, mode, pairs))
    b.close()


def test_batch_high_quality(apg):
    pairs = _pairs(400, mix=[(128, 96, 64, 2), (96, 64, 64, 1)], patch=0.2)
    b = apg.Batch(apg.config_from_mode(2, 64))
    _check(b.process(pairs), _single(apg, 2, pairs))
    b.close()


def test_batch_device_buffers(apg):
    import torch
    from apg_sgm_b200 import _lib
    pairs = _pairs(500, mix=[(160, 96, 64, 2), (200, 120, 128, 1)])
    dev = torch.device("cuda", 0)
    recs, keep, outs = [], [], []
    for L, R, dmax in pairs:
        h, w = L.shape
        dl, dr = torch.from_numpy(L).to(dev), torch.from_numpy(R).to(dev)
        o = {"disparity": torch.empty((h, w), dtype=torch.float32, device=dev),
             "confidence": torch.empty((h, w), dtype=torch.float32, device=dev),
             "invalid_reason": torch.empty((h, w), dtype=torch.uint8, device=dev),
             "reliable_mask": torch.empty((h, w), dtype=torch.uint8, device=dev)}
        keep += [dl, dr]
        outs.append(o)
        recs.append(_lib.Pair(dl.data_ptr(), dr.data_ptr(), w, h, w, 1, dmax, o["disparity"].data_ptr(),
                              o["confidence"].data_ptr(), o["invalid_reason"].data_ptr(),
                              o["reliable_mask"].data_ptr()))
    torch.cuda.synchronize()
    b = apg.Batch(apg.config_from_mode(1, 128))
    b.process_device(recs)
    got = [{k: v.cpu().numpy() for k, v in o.items()} for o in outs]
    _check(got, _single(apg, 1, pairs))
    b.close()


def test_batch_rejects_invalid_pair(apg):
    """A pair with no image is refused before any device work, naming the pair."""
    from apg_sgm_b200 import _lib
    L, R = synth(64, 48, 32)
    out = np.empty((48, 64), np.float32)
    recs = (_lib.Pair * 2)(_lib.Pair(L.ctypes.data, R.ctypes.data, 64, 48, 64, 1, 32, out.ctypes.data, None, None, None),
                           _lib.Pair(None, R.ctypes.data, 64, 48, 64, 1, 32, out.ctypes.data, None, None, None))
    b = apg.Batch(apg.config_from_mode(1, 64))
    assert _lib.lib().apgcu_batch_process(b._h, 2, recs, 0) == 1
    assert "pair 1" in b.last_error
    b.close()
