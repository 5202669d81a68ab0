"""apgcu_right_wta_noalloc: the allocation-free right-image WTA over a caller's cost volume.

Each case runs the engine (apgcu_engine_process) with the raw cost volume kept, uploads that
volume, and calls the no-alloc entry point through the C-ABI twice in a row, on two different
pairs, comparing each result bit for bit with the engine's own right-image disparity.  The
second call checks that the first call's keys do not leak into it.  The file is named to be
collected last, so the entry point also runs after every other test in the process.
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


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_noalloc_right_wta_matches_engine(apg, case):
    import torch
    from apg_sgm_b200._lib import lib

    mode, w, h, dmax, dmin, padded = case
    cfg = apg.config_from_mode(mode, dmax)
    cfg.min_disparity = dmin
    D = cfg.D
    pitch = (D + 63) // 64 * 64 if padded else D
    dev = torch.device("cuda", 0)
    out = torch.empty((h, w), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    for seed in (0, 1):
        L, R = synth(w, h, dmax, cells=5, lo=max(dmin, 0), hi=dmax - 4, seed=40 + seed)
        vol, want = _engine_pair(apg, cfg, L, R)
        d_vol = torch.zeros((h * w, pitch), dtype=torch.int16, device=dev)
        d_vol[:, :D] = torch.from_numpy(vol.reshape(h * w, D).view(np.int16)).to(dev)
        out.fill_(123.0)
        torch.cuda.synchronize()
        rc = lib().apgcu_right_wta_noalloc(C.c_void_p(d_vol.data_ptr()), w, h, dmin, D, pitch, int(cfg.subpixel),
                                           C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert rc == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert same_bits(got, want), (case, seed, int((got != want).sum()))


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
    assert 2049 * 1024 > max_px
