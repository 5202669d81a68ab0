"""On-disk formats (src/image.cpp:62-206): the library's readers and writers against the reference's
own (no GPU).

Writers: the files the library writes equal, byte for byte, those the reference writes for the
same data (8-bit PGM, 16-bit PGM with negative and extreme values, disparity previews with
invalid pixels and small dmax, PFM).  Readers: the library and the reference accept and reject
the same files -- header comments and whitespace variants, maxval bounds, unsupported magics,
truncated samples, big- and little-endian and 3-channel PFM -- and return the same samples.  The
PFM round trip of tests/test_ablation.cpp (test_pfm_io) is repeated.  Without the reference build
only the library-side round trips run.
"""
import numpy as np
import pytest

pytestmark = []


def _need_ref(O):
    if not O.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")


def test_writers_byte_identical(O, apg, tmp_path):
    _need_ref(O)
    rng = np.random.default_rng(3)
    img = rng.integers(0, 256, (37, 53)).astype(np.uint8)
    d16 = rng.integers(-32768, 32767, (21, 30)).astype(np.int16)
    d16[0, :4] = [-1, 0, 32767, -32768]
    disp = rng.uniform(-3, 140, (25, 33)).astype(np.float32)
    disp[0, :5] = [-1.0, 0.0, 127.999, 1e9, np.nan]
    pf = rng.normal(0, 50, (19, 23)).astype(np.float32)
    cases = [("pgm", img, apg.save_pgm, {}), ("pgm16", d16, apg.save_pgm16, {}), ("pfm", pf, apg.save_pfm, {})]
    for kind, a, fn, _ in cases:
        mine, ref = tmp_path / f"m.{kind}", tmp_path / f"r.{kind}"
        fn(mine, a)
        assert O.ref_save(kind, ref, a) == 1
        assert mine.read_bytes() == ref.read_bytes(), kind
    for dmax in (128.0, 0.5, 1.0, 255.0):
        mine, ref = tmp_path / "m.pgm", tmp_path / "r.pgm"
        apg.save_disparity_preview(mine, disp, dmax)
        assert O.ref_save("disparity_preview", ref, disp, dmax) == 1
        assert mine.read_bytes() == ref.read_bytes(), dmax


def _pnm_files(rng):
    g = rng.integers(0, 256, (9, 11)).astype(np.uint8)
    c = rng.integers(0, 256, (7, 5, 3)).astype(np.uint8)
    raw_g, raw_c = g.tobytes(), c.tobytes()
    return {
        "plain_p5": b"P5\n11 9\n255\n" + raw_g,
        "comments_p5": b"P5\n# made by a test\n11 # width\n9\n# maxval next\n255\n" + raw_g,
        "spaces_p5": b"P5 11\t9  255 " + raw_g,
        "crlf_p5": b"P5\r\n11 9\r\n255\r" + raw_g,
        "maxval_100_p5": b"P5\n11 9\n100\n" + raw_g,
        "p6": b"P6\n5 7\n255\n" + raw_c,
        "maxval_256": b"P5\n11 9\n256\n" + raw_g,
        "maxval_0": b"P5\n11 9\n0\n" + raw_g,
        "ascii_p2": b"P2\n11 9\n255\n" + raw_g,
        "short_data": b"P5\n11 9\n255\n" + raw_g[:-1],
        "zero_width": b"P5\n0 9\n255\n",
        "bad_token": b"P5\nab 9\n255\n" + raw_g,
        "trailing_bytes": b"P5\n11 9\n255\n" + raw_g + b"extra",
        "empty": b"",
    }


def test_pnm_reader_matches_reference(O, apg, tmp_path):
    _need_ref(O)
    for name, data in _pnm_files(np.random.default_rng(4)).items():
        p = tmp_path / f"{name}.pnm"
        p.write_bytes(data)
        rc, want = O.ref_load_image(p)
        try:
            got = apg.load_image(p)
        except OSError:
            got = None
        if rc == 1:
            assert got is not None and got.shape == want.shape and np.array_equal(got, want), name
        else:
            assert got is None, name  # the reference fails (or throws) on it: the library rejects it too


def _pfm_files(rng):
    a = rng.normal(0, 10, (6, 8)).astype(np.float32)
    rows_up = a[::-1]
    col3 = np.stack([rows_up, rows_up + 1, rows_up + 2], -1).astype(np.float32)
    return {
        "le": b"Pf\n8 6\n-1.0\n" + rows_up.astype("<f4").tobytes(),
        "be": b"Pf\n8 6\n1.0\n" + rows_up.astype(">f4").tobytes(),
        "comment": b"Pf\n# c1\n8 6 #c2\n-2.5\n" + rows_up.astype("<f4").tobytes(),
        "colour": b"PF\n8 6\n-1.0\n" + col3.astype("<f4").tobytes(),
        "short": b"Pf\n8 6\n-1.0\n" + rows_up.astype("<f4").tobytes()[:-3],
        "bad_tag": b"P7\n8 6\n-1.0\n" + rows_up.astype("<f4").tobytes(),
        "zero_h": b"Pf\n8 0\n-1.0\n",
        "no_scale": b"Pf\n8 6\n",
    }


def test_pfm_reader_matches_reference(O, apg, tmp_path):
    _need_ref(O)
    for name, data in _pfm_files(np.random.default_rng(5)).items():
        p = tmp_path / f"{name}.pfm"
        p.write_bytes(data)
        rc, want = O.ref_load_pfm(p)
        try:
            got = apg.load_pfm(p)
        except OSError:
            got = None
        if rc == 1:
            assert got is not None and np.array_equal(got.view(np.uint32), want.view(np.uint32)), name
        else:
            assert got is None, name


def test_pfm_roundtrip(apg, tmp_path):
    """tests/test_ablation.cpp test_pfm_io: a 16x12 map survives save_pfm / load_pfm."""
    orig = (np.arange(16 * 12, dtype=np.float32).reshape(12, 16) * 0.37 - 5.0).astype(np.float32)
    p = tmp_path / "rt.pfm"
    apg.save_pfm(p, orig)
    back = apg.load_pfm(p)
    assert back.shape == (12, 16)
    assert np.array_equal(back, orig)


def test_pgm_roundtrip_and_errors(apg, tmp_path):
    img = np.random.default_rng(6).integers(0, 256, (13, 17)).astype(np.uint8)
    p = tmp_path / "rt.pgm"
    apg.save_pgm(p, img)
    assert np.array_equal(apg.load_image(p), img)
    with pytest.raises(OSError):
        apg.load_image(tmp_path / "missing.pgm")
    with pytest.raises(ValueError):
        apg.save_pgm(p, np.zeros((3, 4, 3), np.uint8))
