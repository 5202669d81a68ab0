"""The manifest benchmark runner (apg_sgm_b200.benchmark) without a GPU: manifest parsing as the
reference's parse_manifest (apps/benchmark_stereo.cpp:81-125) reads it, ablation presets
(src/ablation.cpp), ablation-id parsing, and the CSV header (the reference runner's own header
where oracle/_ref holds its build)."""
import subprocess

import pytest

from apg_sgm_b200 import benchmark as B


def test_parse_manifest(tmp_path):
    m = tmp_path / "sub" / "m.txt"
    m.parent.mkdir()
    m.write_text("\n".join([
        "# comment",
        "   ",
        "a l.pgm r.pgm g.pfm",
        "b /abs/l.pgm r.pgm g.pfm 64 -8 vis.pgm extra",
        "c l.pgm r.pgm g.pfm 96abc",
        "d l.pgm r.pgm g.pfm xyz 4 v.pgm",
        "e l.pgm r.pgm",
        "\t# indented comment",
        "f ../l.pgm r.pgm g.pfm 32",
    ]) + "\n")
    cs = {c["name"]: c for c in B.parse_manifest(str(m))}
    assert sorted(cs) == ["a", "b", "c", "d", "f"]
    assert (cs["a"]["dmax"], cs["a"]["dmin"], cs["a"]["vis"]) == (128, 0, "")
    assert cs["a"]["left"] == str(m.parent / "l.pgm")
    assert (cs["b"]["left"], cs["b"]["dmax"], cs["b"]["dmin"]) == ("/abs/l.pgm", 64, -8)
    assert cs["b"]["vis"] == str(m.parent / "vis.pgm")
    assert (cs["c"]["dmax"], cs["c"]["dmin"], cs["c"]["vis"]) == (96, 0, "")   # `>> int` stops at "abc"
    assert (cs["d"]["dmax"], cs["d"]["dmin"], cs["d"]["vis"]) == (0, 0, "")    # failed read stores 0
    assert cs["f"]["left"] == str(tmp_path / "l.pgm")


def test_ablation_presets():
    want = {  # use_ad/grad, agg, adaptive, paths, prior, refine
        "A": (0, 0, 0, 4, 0, 0), "B": (1, 0, 0, 4, 0, 0), "C": (1, 1, 0, 4, 0, 0), "D": (1, 1, 1, 4, 0, 0),
        "E": (1, 1, 1, 4, 1, 0), "F": (1, 1, 1, 4, 1, 1), "G": (1, 1, 1, 8, 1, 1)}
    for aid, v in want.items():
        c = B.ablation_config(aid, 96)
        assert (c.use_ad, c.agg_enable, c.adaptive_penalties, c.paths, c.prior_enable, c.refine_enable) == v, aid
        assert c.use_grad == c.use_ad and c.max_disparity == 96 and c.min_disparity == 0
        assert (c.subpixel, c.lr_check, c.median_radius, c.max_fill_gap, c.refine_iterations) == (1, 1, 1, 32, 3)
    assert B.parse_ablations("all") == list("ABCDEFG")
    assert B.parse_ablations(" a, F_refine4 ,zz") == ["A", "F"]


def test_header_matches_reference_runner(O, tmp_path):
    exe = O.HERE / "_ref" / "benchmark_stereo"
    if not exe.exists():
        pytest.skip("reference runner (oracle/_ref/benchmark_stereo) not built")
    (tmp_path / "m.txt").write_text("x missing_l.pgm missing_r.pgm missing.pfm 16\n")
    r = subprocess.run([str(exe), "--manifest", str(tmp_path / "m.txt"), "--output", str(tmp_path / "o.csv")],
                       capture_output=True, text=True)
    # every image is missing: the runner writes its header and no rows
    assert (tmp_path / "o.csv").read_text() == B.HEADER, r.stderr
