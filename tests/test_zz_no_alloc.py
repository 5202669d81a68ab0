"""apgcu_right_wta_noalloc: the allocation-free right-image WTA over a caller's cost volume.

It is for hosts that may not allocate device memory while they run -- a caller with its own fixed
device-memory budget or carved pool, or one whose allocator would synchronise the device -- so it
keeps its per-pixel keys in a static device array instead of a workspace.

Each case runs the engine (apgcu_engine_process) with the raw cost volume kept, uploads that
volume, and calls the no-alloc entry point through the C-ABI twice in a row, on two different
pairs, comparing each result bit for bit (tolerance 0) with the engine's own right-image disparity
and with the oracle's (orc_wta_right, the restatement of wta_right_from_left_volume).  The second
call checks that the first call's keys do not leak into it.  The device's free memory is the same
before and after the two calls: they allocate nothing.  The file is named to be collected last, so
the entry point also runs after every other test in the process; it passes alone in a fresh
process too (one warm-up call loads the module first, as the header asks callers to do).
"""
import ctypes as C

import numpy as np
import pytest

from helpers import same_bits, synth

CASES = [
    # (mode, W, H, dmax, min_disparity, padded pitch)
    (1, 160, 96, 64, 0, False),    # Balanced, subpixel on
    (0, 192, 80, 100, 0, True),    # Fast, volume rows padded to 128
    (1, 130, 70, 48, -6, False),   # negative disparities (reported as -1), ragged width
]


def _engine_pair(apg, cfg, L, R):
    eng = apg.Engine(cfg, debug=apg.DEBUG_RAW_COST)
    eng.process(L, R)
    vol = eng.dump("cost_raw")
    right = eng.dump("disp_right")
    eng.close()
    return vol, right


def _call(lib, d_vol, w, h, dmin, D, pitch, subpixel, out, stream):
    return lib.apgcu_right_wta_noalloc(C.c_void_p(d_vol.data_ptr()), w, h, dmin, D, pitch, int(subpixel),
                                       C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_noalloc_right_wta_matches_engine(apg, O, case):
    import torch
    from apg_sgm_b200._lib import lib

    from helpers import to_oracle

    mode, w, h, dmax, dmin, padded = case
    cfg = apg.config_from_mode(mode, dmax)
    cfg.min_disparity = dmin
    D = cfg.D
    pitch = (D + 63) // 64 * 64 if padded else D
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    # every input, output and expected map is made before the two calls, so that nothing else
    # allocates device memory between the free-memory readings
    frames = []
    for seed in (0, 1):
        L, R = synth(w, h, dmax, cells=5, lo=max(dmin, 0), hi=dmax - 4, seed=40 + seed)
        vol, want = _engine_pair(apg, cfg, L, R)
        oracle_right = O.wta_right(to_oracle(O, cfg), vol)
        d_vol = torch.zeros((h * w, pitch), dtype=torch.int16, device=dev)
        d_vol[:, :D] = torch.from_numpy(vol.reshape(h * w, D).view(np.int16)).to(dev)
        out = torch.full((h, w), 123.0, dtype=torch.float32, device=dev)
        frames.append((d_vol, out, want, oracle_right))
    warm = torch.empty((h, w), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    # warm-up call: the first call on a device may load the library's module into the context
    assert _call(lib(), frames[0][0], w, h, dmin, D, pitch, cfg.subpixel, warm, stream) == 0
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(dev)[0]
    for d_vol, out, _, _ in frames:
        assert _call(lib(), d_vol, w, h, dmin, D, pitch, cfg.subpixel, out, stream) == 0
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info(dev)[0]
    assert free_after == free_before, (free_before, free_after)
    for seed, (_, out, want, oracle_right) in enumerate(frames):
        got = out.cpu().numpy()
        assert same_bits(got, want), (case, seed, int((got != want).sum()))
        assert same_bits(got, oracle_right), (case, seed, int((got != oracle_right).sum()))


def test_noalloc_rejects_sizes_beyond_the_maximum(apg):
    """Sizes beyond the static scratch are refused before anything is launched."""
    from apg_sgm_b200._lib import lib

    fake = C.c_void_p(0x1000)  # never dereferenced: the call returns before touching the device
    max_px = 1 << 21
    assert lib().apgcu_right_wta_noalloc(fake, 2049, 1024, 0, 64, 64, 1, fake, None) == 6  # > 2^21 pixels
    assert lib().apgcu_right_wta_noalloc(fake, 1, 70000, 0, 64, 64, 1, fake, None) == 6    # height > 65535
    assert lib().apgcu_right_wta_noalloc(fake, 64, 64, 0, 1025, 1025, 1, fake, None) == 3  # D > 1024
    assert lib().apgcu_right_wta_noalloc(fake, 64, 64, 0, 64, 63, 1, fake, None) == 2      # pitch < D
    assert lib().apgcu_right_wta_noalloc(None, 64, 64, 0, 64, 64, 1, fake, None) == 1
    assert lib().apgcu_right_wta_noalloc(fake, 64, 64, (1 << 20) + 1, 64, 64, 1, fake, None) == 3  # |d0| too large
    assert lib().apgcu_right_wta_noalloc(fake, 64, 64, -(1 << 20) - 1, 64, 64, 1, fake, None) == 3
    assert 2049 * 1024 > max_px
