"""Page-locked pair loader and the file-fed server (serve_files).

The loader's pairs equal load_image's, its buffers are recycled (the page-locked footprint stops
growing once the pipeline is full), mismatched or missing files fail that pair only, and
serve_files returns, in order, exactly what the single-pair engine gives for each file pair.
"""
import numpy as np
import pytest

from helpers import same_bits, synth

pytestmark = pytest.mark.gpu

KEYS = ("disparity", "confidence", "invalid_reason", "reliable_mask")


def _write_pairs(apg, tmp_path, sizes, seed=40):
    paths, imgs = [], []
    for i, (w, h, d) in enumerate(sizes):
        L, R = synth(w, h, d, seed=seed + i)
        lp, rp = tmp_path / f"l{i}.pgm", tmp_path / f"r{i}.pgm"
        apg.save_pgm(lp, L)
        apg.save_pgm(rp, R)
        paths.append((lp, rp))
        imgs.append((L, R))
    return paths, imgs


def test_loader_reads_and_recycles(apg, tmp_path):
    paths, imgs = _write_pairs(apg, tmp_path, [(160, 96, 64)] * 6)
    ld = apg.Loader(threads=3)
    peak = 0
    for rnd in range(3):
        ts = [ld.submit(*p) for p in paths]
        for t, (L, R) in zip(ts, imgs):
            a, b = ld.wait(t)
            assert np.array_equal(a, L) and np.array_equal(b, R)
            ld.release(t)
        if rnd == 0:
            peak = ld.pinned_bytes
        else:
            assert ld.pinned_bytes == peak  # buffers come back to the pool
    ld.close()


def test_loader_errors_are_per_pair(apg, tmp_path):
    paths, _ = _write_pairs(apg, tmp_path, [(64, 48, 32), (80, 48, 32)])
    ld = apg.Loader(threads=2)
    bad = ld.submit(paths[0][0], paths[1][1])          # sizes differ
    missing = ld.submit(tmp_path / "none.pgm", paths[0][1])
    good = ld.submit(*paths[0])
    with pytest.raises(OSError):
        ld.wait(bad)
    with pytest.raises(OSError):
        ld.wait(missing)
    a, _ = ld.wait(good)
    assert a.shape == (48, 64)
    ld.close()


def test_serve_files_matches_engine(apg, tmp_path):
    sizes = [(160, 96, 64), (200, 120, 64), (160, 96, 64), (128, 64, 64), (200, 120, 64)] * 2
    paths, imgs = _write_pairs(apg, tmp_path, sizes)
    want = []
    for (L, R), (_, _, d) in zip(imgs, sizes):
        e = apg.Engine(apg.config_from_mode(1, d))
        want.append(e.process(L, R))
        e.close()
    srv = apg.Server(slots=3)
    got = list(apg.serve_files(srv, paths, mode=1, max_disparity=64, depth=4))
    srv.close()
    assert [j for j, _, _ in got] == list(range(len(paths)))
    for j, o, lat in got:
        assert lat > 0
        for k in KEYS:
            assert same_bits(o[k], want[j][k]), (j, k)
