"""GPU parity: every stage of the CUDA engine against the CPU oracle, bit for bit.

The oracle (oracle/apg_oracle.c) is pinned to the reference by tests/test_oracle_pins.py.
Integer stages (aux planes, census, ranges, cost volumes, path sums, masks) and float stages
(sub-pixel disparities, confidence, fill, median) are all required to be bit-identical:
tolerance 0, max |delta| = 0.
"""
import numpy as np
import pytest

from helpers import pattern, same_bits, synth, to_oracle

pytestmark = pytest.mark.gpu


def _cases():
    F, B, H = 0, 1, 2
    return [
        # name, mode, (w, h, dmax, dmin), input kind, overrides, debug flags
        ("fast_160x120_d32", F, (160, 120, 32, 0), "synth", {}, 0),
        ("fast_nofusion_160x120_d32", F, (160, 120, 32, 0), "synth", {}, 4),
        ("balanced_97x61_d24", B, (97, 61, 24, 0), "synth", {}, 0),
        ("balanced_160x120_d64", B, (160, 120, 64, 0), "synth", {}, 0),
        ("balanced_100x80_d70", B, (100, 80, 70, 0), "synth", {}, 0),
        ("hq_200x150_d48", H, (200, 150, 48, 0), "synth_patch", {}, 0),
        ("hq_160x120_d32", H, (160, 120, 32, 0), "synth_patch", {}, 0),
        ("negative_range_48x36", B, (48, 36, 8, -4), "noise", {}, 0),
        ("rgb_fast_64x48", F, (64, 48, 16, 0), "rgb", {}, 0),
        ("rgb_balanced_64x48", B, (64, 48, 16, 0), "rgb", {}, 0),
        ("census9x7_balanced_96x64", B, (96, 64, 32, 0), "synth", {"census_type": 0}, 0),
        ("census9x7_fast_96x64", F, (96, 64, 32, 0), "synth", {"census_type": 0}, 0),
        ("path8_balanced_120x90_d40", B, (120, 90, 40, 0), "synth", {"paths": 8}, 0),
        ("fast_260x40_d200", F, (260, 40, 200, 0), "synth", {}, 0),
        ("fast_333x90_d128", F, (333, 90, 128, 0), "synth", {}, 0),
        # the one-byte Fast volume (a padded range of 256): a negative range, 8 paths
        ("fast_300x64_d256", F, (300, 64, 256, 0), "synth", {}, 0),
        ("fast_negative_120x60_d200_min_40", F, (120, 60, 200, -40), "synth", {}, 0),
        ("fast_path8_150x80_d256", F, (150, 80, 256, 0), "synth", {"paths": 8}, 0),
        ("balanced_agg2_80x60", B, (80, 60, 24, 0), "synth", {"agg_iterations": 2}, 0),
        ("balanced_continuous_p2", B, (80, 60, 24, 0), "synth", {"piecewise_p2": 0}, 0),
        ("balanced_min8_max40", B, (120, 60, 40, 8), "synth", {}, 0),
        ("balanced_no_subpixel", B, (80, 60, 24, 0), "synth", {"subpixel": 0}, 0),
        ("balanced_median_r2_nolr", B, (80, 60, 24, 0), "synth", {"median_radius": 2, "lr_check": 0}, 0),
        ("balanced_median_off", B, (80, 60, 24, 0), "synth", {"median_radius": 0}, 0),
        ("checker_odd_33x27", B, (33, 27, 16, 0), "checker", {}, 0),
        ("row_33x1", B, (33, 1, 16, 0), "noise", {}, 0),
        ("column_1x33", B, (1, 33, 16, 0), "noise", {}, 0),
        ("pixel_1x1", F, (1, 1, 16, 0), "noise", {}, 0),
        ("hq_d256_300x100", H, (300, 100, 256, 0), "synth_patch", {}, 0),
        # the aggregated volume at one byte per voxel (a padded range of 256): 4 and 8 paths, a
        # negative range (per-pixel counts in the vertical pass)
        ("balanced_300x64_d256", B, (300, 64, 256, 0), "synth", {}, 0),
        ("path8_balanced_160x80_d256", B, (160, 80, 256, 0), "synth", {"paths": 8}, 0),
        ("balanced_negative_200x60_d200_min_40", B, (200, 60, 200, -40), "synth", {}, 0),
        # refiner wavefront edges: a one-row last band, fewer columns than lanes, a negative range,
        # more passes with a wider random radius
        ("hq_band_edges_70x33", H, (70, 33, 24, 0), "synth_patch", {}, 0),
        ("hq_narrow_20x70", H, (20, 70, 16, 0), "synth_patch", {}, 0),
        ("hq_negative_range_64x48", H, (64, 48, 8, -8), "noise", {}, 0),
        ("hq_refine_5iter_r7", H, (96, 64, 32, 0), "synth_patch", {"refine_iterations": 5, "refine_random_radius": 7}, 0),
    ]


def _inputs(kind, w, h, dmax, dmin):
    if kind == "synth":
        return synth(w, h, dmax, cells=6, lo=max(dmin, 0), hi=max(dmin, 0) + max(1, (dmax - max(dmin, 0)) * 7 // 8))
    if kind == "synth_patch":
        return synth(w, h, dmax, cells=6, lo=0, hi=dmax * 7 // 8, patch=0.2)
    if kind == "rgb":
        l = pattern(w, h, 3, "noise")
        r = np.roll(l, -3, axis=1)
        return l, r
    l = pattern(w, h, 1, kind)
    return l, np.roll(l, -2, axis=1)


CASES = _cases()


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_stage_parity(case, O, apg):
    name, mode, (w, h, dmax, dmin), kind, over, dbg = case
    cfg = apg.config_from_mode(mode, dmax, dmin, **over)
    L, R = _inputs(kind, w, h, dmax, dmin)
    eng = apg.Engine(cfg, debug=apg.DEBUG_RAW_COST | apg.DEBUG_KEEP_SUM | dbg)
    gpu = eng.process(L, R)
    ocfg = to_oracle(O, cfg)
    ora = O.pipeline(ocfg, L, R, stages=True)
    assert ora["status"] == 0
    aux = O.aux(L, R)

    checks = [
        ("left_gray", aux["left"]["gray"]), ("left_gx", aux["left"]["gx"]), ("left_gy", aux["left"]["gy"]),
        ("right_gray", aux["right"]["gray"]), ("right_gx", aux["right"]["gx"]), ("right_gy", aux["right"]["gy"]),
        ("census_left", aux["left"]["census" if cfg.census_type == 1 else "census64"]),
        ("census_right", aux["right"]["census" if cfg.census_type == 1 else "census64"]),
        ("range_min", ora["range_min"]), ("range_max", ora["range_max"]),
        ("cost_raw", ora["cost_raw"]),
    ]
    if cfg.agg_enable:
        checks.append(("cost_agg", ora["cost_agg"]))
    s32 = ora["sgm_sum"]
    assert int(s32[s32 != 0xFFFFFFFF].max(initial=0)) < 0xFFFF
    checks.append(("sgm_sum", np.where(s32 == 0xFFFFFFFF, 0xFFFF, s32).astype(np.uint16)))
    checks += [("disp_wta", ora["disp_wta"]), ("best", ora["best"]), ("second", ora["second"]),
               ("disp_right", ora["disp_right"])]
    if cfg.prior_enable:
        checks.append(("d_prior", ora["d_prior"]))
    if cfg.refine_enable:
        checks.append(("disp_refined", ora["disp_refined"]))
    if cfg.lr_check:
        checks.append(("disp_lr", ora["disp_lr"]))
    checks += [("disp_fill", ora["disp_fill"]), ("disparity", ora["disparity"])]
    for stage, want in checks:
        got = eng.dump(stage)
        if not same_bits(got, want):
            bad = np.argwhere(got != want)
            i = tuple(bad[0]) if len(bad) else None
            pytest.fail(f"{name}: stage {stage} differs at {len(bad)} positions; first {i}: gpu={got[i] if i else None} "
                        f"oracle={want[i] if i else None}")
    # final outputs of the host-copy path
    for k in ("disparity", "confidence", "invalid_reason", "reliable_mask"):
        assert same_bits(gpu[k], ora[k]), f"{name}: final {k} differs"
    assert np.all(np.isfinite(gpu["disparity"]))
    if dmin >= 0:
        # with a non-negative range, a negative disparity is the invalid marker
        neg = gpu["disparity"][gpu["disparity"] < 0]
        assert np.all(neg == -1.0)
    assert np.all((gpu["confidence"] >= 0) & (gpu["confidence"] <= 1))


@pytest.mark.parametrize("w,h,dmax", [(200, 100, 48), (333, 90, 128)])
def test_fast_fused_equals_unfused(apg, w, h, dmax):
    """The census-fused Fast sweeps (tuning fast_fused=1) equal the volume-fed default."""
    L, R = synth(w, h, dmax)
    cfg = apg.config_from_mode(0, dmax)
    fused = apg.Engine(cfg)
    fused.set_tuning("fast_fused", 1)
    a = fused.process(L, R)
    b = apg.Engine(cfg).process(L, R)
    for k in a:
        assert same_bits(a[k], b[k]), k


@pytest.mark.parametrize("mode,w,h,dmax,over", [
    (0, 333, 90, 128, {}), (0, 300, 64, 256, {}), (0, 97, 61, 100, {"min_disparity": -20}),
    (0, 150, 80, 128, {"paths": 8}), (0, 64, 7, 120, {}), (0, 150, 80, 128, {"sgm_split": 2}),
    (1, 300, 64, 256, {}), (1, 150, 80, 128, {}), (1, 160, 90, 256, {"paths": 8}),
    (1, 200, 64, 200, {"min_disparity": -40}), (1, 256, 128, 256, {"hier_enable": 1}), (2, 200, 96, 256, {}),
    (1, 64, 9, 128, {"sgm_split": 2}),
])
def test_cost8_changes_no_result(apg, mode, w, h, dmax, over):
    """The sweeps' volume at one byte per voxel (tuning cost8=2; the default at a padded range of
    256) and at two bytes (cost8=1) give identical maps and path sums, and the byte form takes half
    the volume's bytes: the raw census volume in Fast mode, the aggregated volume otherwise."""
    L, R = synth(w, h, dmax, patch=0.2 if mode == 2 else 0.0, seed=29)
    over = dict(over)
    dmin = over.pop("min_disparity", 0)
    split = over.pop("sgm_split", 0)
    cfg = apg.config_from_mode(mode, dmax, dmin, **over)
    outs, sizes = [], []
    for cost8 in (2, 1):
        e = apg.Engine(cfg, debug=apg.DEBUG_KEEP_SUM)
        e.set_tuning("cost8", cost8)
        e.set_tuning("sgm_split", split)
        o = e.process(L, R)
        o["sgm_sum"] = e.dump("sgm_sum")
        sizes.append(e.allocated_bytes)
        e.close()
        outs.append(o)
    for k in outs[0]:
        assert same_bits(outs[0][k], outs[1][k]), k
    Dp = 128 if dmax - dmin <= 128 else 256
    assert sizes[1] - sizes[0] >= w * h * Dp // 2
    # the default: bytes at 256, two bytes at 128
    e = apg.Engine(cfg, debug=apg.DEBUG_KEEP_SUM)
    e.process(L, R)
    assert e.allocated_bytes == sizes[0 if Dp == 256 else 1]
    e.close()


GOLDEN = {  # tests/test_api_contract.cpp:243-257 of the reference (w, h, invalid, reliable, disp, conf, inv, rel)
    "Odd_Checkerboard": (33, 27, 0, 612, 0x1710451f7eab215, 0xe61822cc0fbe3a38, 0x22081e533cd30004, 0x9ade9d63e4fcae7b),
    "Color_Noise": (32, 24, 0, 720, 0x7e8e0fa784351325, 0x5860e8f479cbe0fd, 0x82f55cc1fd68a695, 0x9db48cb5d76242b5),
    "Negative_Disp_Range": (48, 36, 0, 178, 0x1d8e1d22713fcee9, 0x77f3c5cdbc782a05, 0x8ec5011cb7fb425, 0x3563e2187fb4a965),
}


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("tag", ["Odd_Checkerboard", "Color_Noise"])
def test_golden_fingerprints_gpu(tag, mode, O, apg):
    if tag == "Odd_Checkerboard":
        img = pattern(33, 27, 1, "checker")
    else:
        img = pattern(32, 24, 3, "noise")
    cfg = apg.config_from_mode(mode, 16)
    out = apg.Engine(cfg).process(img, img)
    w, h, inv, rel, dh, ch, ih, rh = GOLDEN[tag]
    assert out["disparity"].shape == (h, w)
    assert int((out["disparity"] < 0).sum()) == inv
    assert int(out["reliable_mask"].sum()) == rel
    assert O.fnv1a64(out["disparity"]) == dh
    assert O.fnv1a64(out["confidence"]) == ch
    assert O.fnv1a64(out["invalid_reason"]) == ih
    assert O.fnv1a64(out["reliable_mask"]) == rh


def test_golden_negative_range_gpu(O, apg):
    img = pattern(48, 36, 1, "noise")
    cfg = apg.config_from_mode(1, 8, -4)
    out = apg.Engine(cfg).process(img, img)
    w, h, inv, rel, dh, ch, ih, rh = GOLDEN["Negative_Disp_Range"]
    assert O.fnv1a64(out["disparity"]) == dh
    assert O.fnv1a64(out["confidence"]) == ch
    assert O.fnv1a64(out["invalid_reason"]) == ih
    assert O.fnv1a64(out["reliable_mask"]) == rh


@pytest.mark.parametrize("mode,spec", [(1, (640, 480, 64, 8, 4, 60)), (0, (1280, 720, 128, 12, 0, 120))])
def test_baseline_workloads_match_oracle(mode, spec, O, apg):
    """The benchmark workloads themselves (640x480 D64 Balanced, 1280x720 D128 Fast)."""
    from apg_sgm_b200 import synthetic as S
    L, R, _ = S.make_pair(S.PairSpec(*spec), S.SEED_BASE)
    cfg = apg.config_from_mode(mode, spec[2])
    gpu = apg.Engine(cfg).process(L, R)
    ora = O.pipeline(to_oracle(O, cfg), L, R)
    for k in ("disparity", "confidence", "invalid_reason", "reliable_mask"):
        assert same_bits(gpu[k], ora[k]), k


@pytest.mark.parametrize("mode,w,h,dmax", [(0, 160, 96, 64), (1, 150, 90, 48), (2, 128, 96, 64)])
def test_session_frame_stats_match_reference(apg, O, mode, w, h, dmax):
    """PipelineStats counters and ratios of the session equal the reference session's
    (src/pipeline.cpp:650-707): counted on the device, float32 ratios."""
    if not O.ref_available():
        pytest.skip("oracle/_ref not built")
    L, R = synth(w, h, dmax, patch=0.2 if mode == 2 else 0.0, seed=11)
    name = {0: "fast", 1: "balanced", 2: "high_quality"}[mode]
    sess = apg.StereoSession(mode=name, max_disparity=dmax, memory_policy="bounded_reuse")
    res = sess.process(L, R)
    ref = O.RefSession(O.config(mode, dmax, volume_backend=2)).process(L, R)
    assert ref["status"] == 0
    for k in ("disparity", "confidence", "invalid_reason", "reliable_mask"):
        assert same_bits(getattr(res, k), ref[k]), k
    st, rs = res.stats, ref["stats"]
    for k in ("valid_pixels", "reliable_pixels", "unreliable_pixels", "refine_changed_pixels", "prior_support_count"):
        assert getattr(st, k) == int(rs[k]), (k, getattr(st, k), rs[k])
    for k in ("valid_disparity_ratio", "reliable_ratio", "unreliable_ratio", "refine_changed_ratio", "lr_fail_ratio",
              "mean_search_width", "mean_geometry_width"):
        assert getattr(st, k) == rs[k], (k, getattr(st, k), rs[k])


@pytest.mark.parametrize("mode,tile", [(1, 64), (1, 256), (0, 256), (2, 128)])
def test_cost_tile_changes_no_result(apg, mode, tile):
    """The cost kernel's tile width (tuning key cost_tile) changes no output."""
    L, R = synth(300, 90, 96, patch=0.2 if mode == 2 else 0.0, seed=21)
    cfg = apg.config_from_mode(mode, 96)
    a = apg.Engine(cfg).process(L, R)
    e = apg.Engine(cfg)
    e.set_tuning("cost_tile", tile)
    b = e.process(L, R)
    for k in a:
        assert same_bits(a[k], b[k]), k


@pytest.mark.parametrize("mode,dmin", [(0, 0), (1, 0), (1, 8)])
def test_range_dump_without_debug(apg, mode, dmin):
    """Frames without a prior use the default ranges in closed form and skip writing the range
    planes; a later dump writes them on demand: [d0, max(min(dmax, x + 1), d0)) per column."""
    w, h, dmax = 150, 20, 64
    L, R = synth(w, h, dmax, seed=3)
    e = apg.Engine(apg.config_from_mode(mode, dmax, dmin))
    e.process(L, R)
    rmin, rmax = e.dump("range_min"), e.dump("range_max")
    e.close()
    x = np.arange(w)
    want_max = np.maximum(np.minimum(dmax, x + 1), dmin).astype(np.int16)
    assert (rmin == dmin).all()
    assert (rmax == want_max[None, :]).all()


@pytest.mark.parametrize("mode,w,h,dmax,over", [
    (0, 200, 100, 48, {}), (1, 333, 90, 128, {}), (1, 150, 80, 200, {}), (1, 120, 90, 40, {"paths": 8}),
    (2, 160, 96, 64, {}), (1, 97, 61, 24, {"min_disparity": -6}), (0, 64, 7, 16, {}),
])
def test_sgm_split_changes_no_result(apg, mode, w, h, dmax, over):
    """The last sweep split over two warps per chain (tuning sgm_split=2) and the one-warp form
    (sgm_split=1) give identical maps and path sums, for every range width and both path counts."""
    L, R = synth(w, h, dmax, patch=0.2 if mode == 2 else 0.0, seed=23)
    over = dict(over)
    dmin = over.pop("min_disparity", 0)
    cfg = apg.config_from_mode(mode, dmax, dmin, **over)
    outs = []
    for split in (1, 2):
        e = apg.Engine(cfg, debug=apg.DEBUG_KEEP_SUM)
        e.set_tuning("sgm_split", split)
        o = e.process(L, R)
        o["sgm_sum"] = e.dump("sgm_sum")
        e.close()
        outs.append(o)
    for k in outs[0]:
        assert same_bits(outs[0][k], outs[1][k]), k
