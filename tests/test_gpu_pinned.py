"""Page-locked caller buffers: the same results as pageable ones.

Host images in page-locked memory go up by DMA from where they lie (no staging copy), and
page-locked result arrays take the device copies directly.  Every entry point that takes host
buffers -- the session C API (through StereoSession), the engine, the batched form and the served
form -- must give bit-identical maps either way, strided images included.
"""
import numpy as np
import pytest

from helpers import same_bits, synth

pytestmark = pytest.mark.gpu

KEYS = ("disparity", "confidence", "invalid_reason", "reliable_mask")


def _pinned(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()


def _pinned_strided(a, pad=13):
    """a as a row-padded view into one page-locked buffer (stride w + pad)."""
    h, w = a.shape
    buf = _pinned(np.zeros((h, w + pad), a.dtype))
    buf[:, :w] = a
    return buf[:, :w]


def _pinned_out(h, w):
    return {"disparity": _pinned(np.zeros((h, w), np.float32)), "confidence": _pinned(np.zeros((h, w), np.float32)),
            "invalid_reason": _pinned(np.zeros((h, w), np.uint8)), "reliable_mask": _pinned(np.zeros((h, w), np.uint8))}


@pytest.mark.parametrize("mode,w,h,dmax", [(1, 320, 200, 128), (0, 256, 96, 64), (2, 200, 120, 64)])
def test_engine_pinned_inputs_match(apg, mode, w, h, dmax):
    L, R = synth(w, h, dmax, patch=0.2 if mode == 2 else 0.0, seed=81)
    e = apg.Engine(apg.config_from_mode(mode, dmax))
    want = e.process(L, R)
    got = e.process(_pinned(L), _pinned(R))
    got_s = e.process(_pinned_strided(L), _pinned_strided(R))
    e.close()
    for k in KEYS:
        assert same_bits(got[k], want[k]), k
        assert same_bits(got_s[k], want[k]), k


def test_session_pinned_inputs_match(apg):
    L, R = synth(320, 180, 128, seed=82)
    s = apg.StereoSession(mode="balanced", max_disparity=128)
    want = s.process(L, R)
    got = s.process(_pinned(L), _pinned(R))
    for k in ("disparity", "confidence"):
        assert same_bits(getattr(got, k), getattr(want, k)), k


def test_batch_pinned_buffers_match(apg):
    sizes = [(160, 96, 64), (200, 120, 128), (256, 64, 192)]
    pairs = [synth(w, h, d, seed=83 + i) for i, (w, h, d) in enumerate(sizes)]
    b = apg.Batch(apg.config_from_mode(1, 128))
    want = b.process([(L, R, d) for (L, R), (_, _, d) in zip(pairs, sizes)])
    outs = [_pinned_out(h, w) for (w, h, _) in sizes]
    got = b.process([(_pinned(L), _pinned(R), d) for (L, R), (_, _, d) in zip(pairs, sizes)], out=outs)
    # mixed: pageable outputs after page-locked ones on the same engines
    again = b.process([(L, R, d) for (L, R), (_, _, d) in zip(pairs, sizes)])
    b.close()
    for i in range(len(sizes)):
        assert got[i] is outs[i]
        for k in KEYS:
            assert same_bits(got[i][k], want[i][k]), (i, k)
            assert same_bits(again[i][k], want[i][k]), (i, k)


def test_server_pinned_buffers_match(apg):
    sizes = [(160, 96, 64), (200, 120, 128)]
    pairs = [synth(w, h, d, seed=90 + i) for i, (w, h, d) in enumerate(sizes)]
    want = []
    for (L, R), (_, _, d) in zip(pairs, sizes):
        e = apg.Engine(apg.config_from_mode(1, d))
        want.append(e.process(L, R))
        e.close()
    srv = apg.Server(slots=2)
    tickets = []
    for i, ((L, R), (w, h, d)) in enumerate(zip(pairs, sizes)):
        o = _pinned_out(h, w)
        tickets.append((i, o, srv.submit(_pinned(L), _pinned(R), mode=1, max_disparity=d, out=o)))
    for i, o, t in tickets:
        got, _ = srv.wait(t)
        for k in KEYS:
            assert same_bits(got[k], want[i][k]), (i, k)
    srv.close()


def test_session_results_are_views_of_pooled_blocks(apg):
    """StereoSession.process returns arrays over the page-locked block the device copies landed in
    (no copy).  A block is not reused while any array of its frame is alive, and is reused once
    they are all gone; every frame equals the engine's."""
    L1, R1 = synth(160, 96, 32, seed=1)
    L2, R2 = synth(160, 96, 32, seed=2)
    s = apg.StereoSession(mode="fast", max_disparity=32, memory_policy="bounded_reuse")
    a = s.process(L1, R1)
    a_disp = a.disparity.copy()
    b = s.process(L2, R2)
    assert a.disparity.ctypes.data != b.disparity.ctypes.data
    assert np.array_equal(a.disparity.view(np.uint32), a_disp.view(np.uint32))
    p = b.disparity.ctypes.data
    del b
    c = s.process(L2, R2)
    assert c.disparity.ctypes.data == p
    want = apg.Engine(apg.config_from_mode(0, 32)).process(L2, R2)
    for k in ("disparity", "confidence", "invalid_reason", "reliable_mask"):
        assert np.array_equal(np.ascontiguousarray(getattr(c, k)).view(np.uint8),
                              np.ascontiguousarray(want[k]).view(np.uint8)), k
    conf = c.confidence
    del c
    assert conf.base is not None and np.all((conf >= 0) & (conf <= 1))  # the view keeps its block
