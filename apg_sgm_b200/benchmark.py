"""Manifest benchmark runner on the GPU path (apps/benchmark_stereo.cpp of the reference).

    python -m apg_sgm_b200.benchmark --manifest cases.txt [--ablation all] [--output results.csv]
        [--save_disp DIR] [--warmup 2] [--repeat 5] [--hierarchical ...] [--subpixel-method M]
        [--subpixel-param P] [--inpaint-method M] [--inpaint-gap N]

Manifest: one case per line, `name left right gt [dmax [dmin [vis]]]`; blank lines and lines
starting with '#' are skipped, relative paths are taken from the manifest's directory
(parse_manifest, apps/benchmark_stereo.cpp:81-125).  For every case and ablation preset A-G
(make_ablation_config, src/ablation.cpp) the pair runs `--warmup` times, then `--repeat` timed
times through a BoundedReuse session; the median run by host time is reported, its accuracy
scored against the ground truth with evaluate_stereo on the GPU.  The CSV has the reference's
columns in the reference's order and number formats, the prior presets' support-match block from
the engine's supports (evaluate_supports on the GPU), and the scopes' telemetry columns with
--subpixel-telem / --inpaint-telem (zeros without, as the reference writes them).  `backend` is
`cuda`.
"""
from __future__ import annotations

import argparse
import os
import re
import sys
import time
from pathlib import Path

import numpy as np

from . import (ExperimentalInpaintScope, ExperimentalSubpixelScope, StereoSession, config_from_mode, evaluate_stereo,
               evaluate_supports, load_image, load_pfm, save_disparity_preview, save_pfm, save_pgm)
from ._lib import PipelineConfig

ABLATIONS = ["A", "B", "C", "D", "E", "F", "G"]
_DESC = {"A": "Census + 4SGM", "B": "Census+AD+Grad + 4SGM", "C": "Census+AD+Grad + Cross + 4SGM",
         "D": "Census+AD+Grad + Cross + AdaptiveP2 + 4SGM", "E": "AdaptiveP2 + Prior + 4SGM",
         "F": "Prior + Refiner + 4SGM", "G": "Prior + Refiner + 8SGM (HQ)"}
_LONG = {"A_CENSUS4": "A", "B_MULTICOST4": "B", "C_CROSS4": "C", "D_ADAPTIVE4": "D", "E_PRIOR4": "E",
         "F_REFINE4": "F", "G_HQ8": "G"}

HEADER = (
    "backend,threads,effective_threads,warmup,repeat,build_type,"
    "case,ablation_id,ablation_name,cost,cross,p2,prior,refine,paths,w,h,dmax,"
    "epe,bad_0_5,bad_1_0,bad_2_0,bad_3_0,kitti_d1_all,kitti_d1_noc,valid_ratio,lr_fail_ratio,edge_epe,nonedge_epe,"
    "recall_all,recall_matchable,recall_visible,range_vis_eval_px,range_vis_in_px,range_mat_eval_px,range_mat_in_px,"
    "prior_miss_vis_count,prior_miss_edge_pct,prior_miss_nonedge_pct,"
    "prior_supports,support_p05,support_p1,support_p2,support_p1_vis,support_pvis_05,support_pvis_1,support_pvis_2,"
    "support_gt_valid,support_visible,support_correct_05,support_correct_1,support_correct_2,"
    "support_visible_correct_05,support_visible_correct_1,support_visible_correct_2,"
    "support_visible_gt_cells,support_correct_visible_cells,"
    "support_mae,support_mae_vis,grid_recall_1,"
    "mean_search_width,mean_geom_width,geom_reduction_ratio,prior_incremental_reduction,total_reduction_ratio,"
    "cost_bytes,cost32_bytes,peak_bytes,"
    "reliable_ratio,unreliable_ratio,refine_changed_ratio,refine_epe_delta,post_epe_delta,total_epe_delta,"
    "time_total_ms,time_aux_ms,time_prior_ms,time_cost_ms,time_right_wta_ms,time_cross_ms,time_sgm_ms,time_wta_ms,"
    "time_confidence_ms,time_refine_ms,time_post_ms,"
    + "".join(f"{p}_pixels,{p}_valid_est_pixels,{p}_valid_ratio,{p}_epe,{p}_bad05,{p}_bad10,{p}_bad20,{p}_bad30,{p}_d1,"
              .replace("all_pixels", "all_gt_pixels")
              for p in ("all", "noc", "occ", "bnd", "nonbnd", "lowtex", "hightex"))
    + "peak_workspace_bytes,retained_workspace_bytes,"
    "avg_states_per_pixel,coarse_valid_ratio,fallback_pixel_ratio,full_range_pixel_ratio,"
    "subpixel_method,subpixel_param,subpixel_candidate_px,subpixel_applied_px,subpixel_applied_ratio,"
    "subpixel_degenerate_count,subpixel_clamped_count,subpixel_clamped_ratio,subpixel_neg_curv_count,"
    "subpixel_mean_abs_delta,subpixel_p50_abs_delta,subpixel_p95_abs_delta,"
    "inpaint_method,inpaint_gap,inpaint_total_holes,inpaint_filled_holes,inpaint_fill_ratio,"
    "inpaint_occ_two_sided,inpaint_occ_left_only,inpaint_occ_right_only,inpaint_occ_unfilled,"
    "inpaint_mism_two_sided,inpaint_mism_left_only,inpaint_mism_right_only,inpaint_mism_unfilled,"
    "inpaint_reclassified_shadow,inpaint_hit_max_gap\n")

_SP_STR = {0: "legacy", 1: "curv_gate", 2: "conf_gate", 3: "stabilized"}
_SP_PARSE = {"legacy": 0, "A": 0, "a": 0, "curv_gate": 1, "curv": 1, "B": 1, "b": 1, "conf_gate": 2, "conf": 2,
             "C": 2, "c": 2, "stabilized": 3, "stab": 3, "D": 3, "d": 3}
_IP_STR = {0: "legacy", 1: "shadow_reclass"}
_IP_PARSE = {"legacy": 0, "A": 0, "a": 0, "shadow_reclass": 1, "shadow": 1, "C": 1, "c": 1}
_FB_PARSE = {"full_range": 1, "FULL_RANGE": 1, "full": 1, "nearest_valid": 0, "NEAREST_VALID": 0, "nearest": 0,
             "expanded_radius": 2, "EXPANDED_RADIUS": 2, "expanded": 2}


def ablation_config(aid: str, max_disparity: int = 128) -> PipelineConfig:
    """make_ablation_config (src/ablation.cpp): the default configuration with the preset's
    cost terms, aggregation, penalties, paths, prior and refiner."""
    c = config_from_mode(1, max_disparity)
    c.min_disparity, c.max_disparity = 0, max_disparity
    c.subpixel, c.lr_check, c.post_lr_max_diff, c.median_radius, c.max_fill_gap = 1, 1, 1, 1, 32
    k = "ABCDEFG".index(aid)
    c.use_ad = c.use_grad = 1 if k >= 1 else 0
    c.agg_enable = 1 if k >= 2 else 0
    c.agg_iterations = 1
    c.adaptive_penalties = 1 if k >= 3 else 0
    c.paths = 8 if k == 6 else 4
    c.prior_enable = 1 if k >= 4 else 0
    c.refine_enable = 1 if k >= 5 else 0
    c.refine_iterations = 3
    return c


def parse_ablations(arg: str):
    if arg in ("all", "ALL"):
        return list(ABLATIONS)
    out = []
    for tok in arg.split(","):
        t = tok.strip().upper()
        if not t:
            continue
        if t in ABLATIONS or t in _LONG:
            out.append(_LONG.get(t, t))
        else:
            print(f"Warning: unrecognized ablation ID: {tok.strip()}", file=sys.stderr)
    return out


def parse_manifest(path: str):
    """apps/benchmark_stereo.cpp:81-125: name left right gt [dmax [dmin [vis]]]."""
    base = Path(path).parent
    cases = []
    for line in Path(path).read_text().splitlines():
        s = line.lstrip(" \t\r\n")
        if not s or s[0] == "#":
            continue
        tok = s.split()
        if len(tok) < 4:
            continue
        c = {"name": tok[0], "left": tok[1], "right": tok[2], "gt": tok[3], "dmax": 128, "dmin": 0, "vis": ""}
        # `iss >> dmax >> dmin >> vis` after the four names: an int field reads the longest integer
        # prefix; a field with none stores 0 and ends the line (the stream has failed)
        rest = s.split(None, 4)[4] if len(tok) > 4 else ""
        ok = True
        for key in ("dmax", "dmin"):
            r = rest.lstrip()
            if not r:
                ok = False
                break
            mm = re.match(r"[+-]?\d+", r)
            if not mm:
                c[key] = 0
                ok = False
                break
            c[key] = int(mm.group(0))
            rest = r[mm.end():]
        if ok and rest.strip():
            c["vis"] = rest.split()[0]
        for k in ("left", "right", "gt", "vis"):
            if c[k] and not os.path.isabs(c[k]):
                c[k] = os.path.normpath(str(base / c[k]))
        cases.append(c)
    return cases


def _f(v, p):
    return f"{float(v):.{p}f}"


def _region(r) -> str:
    return (f"{r.total_pixels},{r.valid_est_pixels},{_f(r.valid_ratio, 4)},{_f(r.epe, 4)},{_f(r.bad_0_5, 4)},"
            f"{_f(r.bad_1_0, 4)},{_f(r.bad_2_0, 4)},{_f(r.bad_3_0, 4)},{_f(r.d1, 4)},")


def run(args) -> int:
    cases = parse_manifest(args.manifest)
    if not cases:
        print(f"Error: no valid test cases found in manifest: {args.manifest}", file=sys.stderr)
        return 1
    ids = parse_ablations(args.ablation)
    if not ids:
        print("Error: no valid ablation configurations selected.", file=sys.stderr)
        return 1
    sp_method, ip_method = _SP_PARSE[args.subpixel_method], _IP_PARSE[args.inpaint_method]
    out = Path(args.output)
    out.parent.mkdir(parents=True, exist_ok=True)
    if args.save_disp:
        Path(args.save_disp).mkdir(parents=True, exist_ok=True)
    rows = [HEADER]
    for c in cases:
        print(f"\n=== Dataset Case: {c['name']} (dmax={c['dmax']}, dmin={c['dmin']}) ===")
        try:
            left, right = load_image(c["left"]), load_image(c["right"])
        except OSError:
            print(f"Failed to load images of {c['name']}", file=sys.stderr)
            continue
        try:
            gt = load_pfm(c["gt"])
            has_gt = True
        except OSError:
            gt, has_gt = None, False
            print(f"Note: could not load GT PFM ({c['gt']}), will report metrics as N/A")
        vis = None
        if c["vis"]:
            try:
                vis = load_image(c["vis"])
                if vis.ndim == 3:
                    vis = np.ascontiguousarray(vis[..., 0])  # vis_mask.at(x, y) reads channel 0
            except OSError:
                vis = None
        h, w = left.shape[:2]
        for aid in ids:
            cfg = ablation_config(aid, c["dmax"])
            cfg.min_disparity, cfg.max_disparity = c["dmin"], c["dmax"]
            cfg.num_threads = args.threads
            if args.hierarchical:
                cfg.hier_enable, cfg.hier_radius = 1, args.hierarchical_radius
                cfg.hier_fallback = _FB_PARSE[args.hierarchical_fallback]
                cfg.hier_coarse_cross_agg = 0 if args.hierarchical_no_cross else 1
                cfg.hier_coarse_fill_holes = 0 if args.hierarchical_no_fill else 1
                cfg.hier_adaptive_radius = 1 if args.hierarchical_adaptive else 0
                cfg.hier_confidence_threshold = args.hierarchical_confidence_threshold
                cfg.hier_expanded_radius = args.hierarchical_expanded_radius
            cfg.max_fill_gap = args.inpaint_gap
            with ExperimentalSubpixelScope(sp_method, args.subpixel_param, args.subpixel_telem), \
                    ExperimentalInpaintScope(ip_method, args.inpaint_gap, args.inpaint_telem):
                sess = StereoSession(config=cfg, memory_policy="bounded_reuse")
                for _ in range(args.warmup):
                    sess.process(left, right)
                _reset_telemetry(args)  # counters of the timed runs only (benchmark_stereo.cpp:545-550)
                samples = []
                for _ in range(args.repeat):
                    t0 = time.perf_counter()
                    res = sess.process(left, right)
                    samples.append(((time.perf_counter() - t0) * 1000.0, res, sess.hierarchical_telemetry))
                tel = (ExperimentalSubpixelScope.current_telemetry(), ExperimentalInpaintScope.current_telemetry())
                samples.sort(key=lambda s: s[0])
                total_ms, res, htel = samples[args.repeat // 2]
                st = res.stats
                m = sm = None
                if has_gt:
                    # the frame's ranges and refine maps come from an engine run of the same pair
                    from . import Engine
                    e = Engine(cfg)
                    e.process(left, right)
                    rng = (e.dump("range_min"), e.dump("range_max")) if (cfg.prior_enable or args.hierarchical) else None
                    before = e.dump("disp_wta") if cfg.refine_enable else None
                    after = e.dump("disp_refined") if cfg.refine_enable else None
                    sup = e.supports() if cfg.prior_enable else None
                    e.close()
                    m = evaluate_stereo(res.disparity, gt, rng, before, after, vis, 1e5, left)
                    if sup is not None and len(sup[0]) > 0:  # has_supports: the prior's list is not empty
                        sm = evaluate_supports(sup, gt, vis, 1e5)
            rows.append(_row(args, c, aid, cfg, w, h, m, sm, st, total_ms, htel, sp_method, ip_method, tel))
            z = m if m is not None else None
            print(f"[{aid}] {_DESC[aid]:32s} | EPE: {(z.epe if z else -1.0):6.3f} | "
                  f"Bad2.0: {(z.bad_2_0 if z else -1.0):5.1f}% | D1-all: {(z.kitti_d1_all if z else -1.0):5.1f}% | "
                  f"D_bar: {st.mean_search_width:4.1f} | Time: {total_ms:6.2f} ms (SGM: {st.timing.sgm_ms:.2f} ms)")
            if args.save_disp:
                prefix = os.path.join(args.save_disp, f"{c['name']}_{aid}")
                save_pfm(prefix + "_disp.pfm", res.disparity)
                save_disparity_preview(prefix + "_disp.pgm", res.disparity, float(c["dmax"]))
                if cfg.prior_enable and has_gt and m is not None and m.has_range:
                    g = np.nan_to_num(gt, nan=-1.0, posinf=-1.0)
                    xr = np.arange(w)[None, :] - np.round(g).astype(np.int64)
                    vis_ok = (vis >= 200) if vis is not None else ((xr >= 0) & (xr < w))
                    miss = (g >= 0) & vis_ok & ((g < rng[0]) | (g >= rng[1]))
                    save_pgm(prefix + "_miss.pgm", np.where(miss, 255, 0).astype(np.uint8))
    out.write_text("".join(rows))
    print(f"\nBenchmark complete. Results written to: {out}")
    return 0


def _reset_telemetry(args):
    from ._lib import lib
    lib().apgcu_reset_telemetry(int(args.subpixel_telem), int(args.inpaint_telem))


def _per_run(tel, repeat, sp_on, ip_on):
    """The timed runs' telemetry divided by the repeat count, each counter with integer division
    and the |delta| sum in double, as benchmark_stereo.cpp:588-600 and 673-688 do."""
    from . import InpaintTelemetry, SubpixelTelemetry
    from ._lib import InpaintTelemetryRec, SubpixelTelemetryRec
    sp, ip = tel
    if not sp_on:
        sp = SubpixelTelemetry(SubpixelTelemetryRec())
    if not ip_on:
        ip = InpaintTelemetry(InpaintTelemetryRec())
    if repeat > 1:
        for k in ("candidate_pixels", "applied_pixels", "degenerate_count", "clamped_count",
                  "negative_curvature_count"):
            setattr(sp, k, getattr(sp, k) // repeat)
        sp.sum_abs_delta = sp.sum_abs_delta / repeat
        sp.delta_buckets = [v // repeat for v in sp.delta_buckets]
        for k in ("total_invalid_pixels", "classified_occ_pixels", "classified_mismatch_pixels", "hit_max_gap_pixels",
                  "reclassified_shadow_pixels", "invalid_runs_count", "invalid_runs_truncated"):
            setattr(ip, k, getattr(ip, k) // repeat)
        ip.route_counts = [v // repeat for v in ip.route_counts]
        ip.run_length_buckets = [v // repeat for v in ip.run_length_buckets]
    return sp, ip


def _row(args, c, aid, cfg, w, h, m, sm, st, total_ms, htel, sp_method, ip_method, tel) -> str:
    has = m is not None
    z = lambda k: getattr(m, k) if has else 0.0  # noqa: E731
    cost = "Census+AD+Grad" if (cfg.use_ad or cfg.use_grad) else "Census"
    cross = f"On({cfg.agg_iterations})" if cfg.agg_enable else "Off"
    r = (f"cuda,{args.threads},{args.threads or 1},{args.warmup},{args.repeat},Release,{c['name']},{aid},"
         f"\"{_DESC[aid]}\",{cost},{cross},{'Adaptive' if cfg.adaptive_penalties else 'Fixed'},"
         f"{'On' if cfg.prior_enable else 'Off'},{'On' if cfg.refine_enable else 'Off'},{cfg.paths},{w},{h},"
         f"{c['dmax']},")
    r += ",".join(_f(z(k), 4) for k in ("epe", "bad_0_5", "bad_1_0", "bad_2_0", "bad_3_0", "kitti_d1_all",
                                         "kitti_d1_noc", "valid_ratio", "lr_fail_ratio", "edge_epe",
                                         "nonedge_epe")) + ","
    if cfg.prior_enable and has and m.has_range:
        r += (f"{_f(m.range_recall_all, 4)},{_f(m.range_recall_matchable, 4)},{_f(m.range_recall_visible, 4)},"
              f"{m.range_visible_eval_pixels},{m.range_visible_in_pixels},{m.range_matchable_eval_pixels},"
              f"{m.range_matchable_in_pixels},{m.prior_miss_visible_count},"
              f"{_f(np.float32(m.prior_miss_edge_ratio) * np.float32(100.0), 2)},"
              f"{_f(np.float32(m.prior_miss_nonedge_ratio) * np.float32(100.0), 2)},")
    else:
        r += "N/A,N/A,N/A,0,0,0,0,0,0.00,0.00,"
    if cfg.prior_enable and has and sm is not None:
        r += (f"{st.prior_support_count},"
              + ",".join(_f(getattr(sm, k), 4) for k in ("precision_all_05", "precision_all_1", "precision_all_2",
                                                         "precision_vis_1", "precision_vis_05", "precision_vis_1",
                                                         "precision_vis_2")) + ","
              + ",".join(str(getattr(sm, k)) for k in ("gt_valid", "visible", "correct_05", "correct_1", "correct_2",
                                                       "visible_correct_05", "visible_correct_1", "visible_correct_2",
                                                       "visible_gt_cells", "correct_visible_cells")) + ","
              + ",".join(_f(getattr(sm, k), 4) for k in ("mae_all", "mae_visible", "grid_recall_1")) + ",")
    else:
        r += f"{st.prior_support_count},0.0,0.0,0.0,0.0,0.0,0.0,0.0,0,0,0,0,0,0,0,0,0,0,0.0,0.0,0.0,"
    D = cfg.max_disparity - cfg.min_disparity
    geom = 1.0 - st.mean_geometry_width / D if D > 0 else 0.0
    incr = (1.0 - st.mean_search_width / st.mean_geometry_width) if st.mean_geometry_width > 0 else 0.0
    total = 1.0 - st.mean_search_width / D if D > 0 else 0.0
    r += (f"{_f(st.mean_search_width, 2)},{_f(st.mean_geometry_width, 2)},{_f(geom, 4)},"
          f"{_f(incr if cfg.prior_enable else 0.0, 4)},{_f(total, 4)},{st.cost_bytes},0,{st.estimated_peak_bytes},"
          f"{_f(st.reliable_ratio, 4)},{_f(st.unreliable_ratio, 4)},")
    ref = has and m.has_refine_stats
    r += ",".join(_f(getattr(m, k) if ref else 0.0, 4)
                  for k in ("refine_changed_ratio", "refine_epe_delta", "post_epe_delta", "total_epe_delta")) + ","
    t = st.timing
    r += ",".join(_f(v, 2) for v in (total_ms, t.aux_ms, t.prior_ms, t.cost_ms, t.right_wta_ms, t.cross_ms, t.sgm_ms,
                                      t.wta_ms, t.confidence_ms, t.refine_ms, t.post_ms)) + ","
    if has:
        for reg in ("reg_all", "reg_noc", "reg_occ", "reg_boundary", "reg_non_boundary", "reg_low_texture",
                    "reg_high_texture"):
            r += _region(getattr(m, reg))
    else:
        r += "0,0,0.0000,0.0000,0.0000,0.0000,0.0000,0.0000,0.0000," * 7
    peak = st.peak_workspace_bytes if st.peak_workspace_bytes > 0 else st.estimated_peak_bytes
    r += f"{peak},{st.retained_workspace_bytes},"
    if args.hierarchical:
        hv = (htel["avg_states_per_pixel"], htel["coarse_valid_ratio"], htel["fallback_pixel_ratio"],
              htel["full_range_pixel_ratio"])
    else:
        hv = (st.mean_search_width, 0.0, 0.0, 0.0)
    r += ",".join(_f(v, 4) for v in hv) + ","
    sp, ip = _per_run(tel, args.repeat, args.subpixel_telem, args.inpaint_telem)
    r += (f"{_SP_STR[sp_method]},{_f(args.subpixel_param, 4)},{sp.candidate_pixels},{sp.applied_pixels},"
          f"{_f(sp.applied_ratio(), 4)},{sp.degenerate_count},{sp.clamped_count},{_f(sp.clamped_ratio(), 4)},"
          f"{sp.negative_curvature_count},{_f(sp.mean_abs_delta(), 4)},{_f(sp.p50_abs_delta(), 4)},"
          f"{_f(sp.p95_abs_delta(), 4)},")
    rc = ip.route_counts
    r += (f"{_IP_STR[ip_method]},{args.inpaint_gap},{ip.total_invalid_pixels},{ip.total_filled_pixels()},"
          f"{_f(ip.fill_ratio(), 4)},{rc[1]},{rc[2]},{rc[3]},{ip.occ_unfilled_pixels()},{rc[7]},{rc[8]},{rc[9]},"
          f"{ip.mismatch_unfilled_pixels()},{ip.reclassified_shadow_pixels},{ip.hit_max_gap_pixels}\n")
    return r


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--manifest", required=True)
    ap.add_argument("--ablation", "--modes", dest="ablation", default="all")
    ap.add_argument("--output", default="results/ablation.csv")
    ap.add_argument("--save_disp", default="")
    ap.add_argument("--warmup", type=lambda v: max(0, int(v)), default=2)
    ap.add_argument("--repeat", type=lambda v: max(1, int(v)), default=5)
    ap.add_argument("--threads", type=lambda v: max(0, int(v)), default=0)
    ap.add_argument("--backend", default="auto", choices=["auto", "dense", "packed", "cuda"],
                    help="accepted for compatibility: every backend runs the CUDA engine")
    ap.add_argument("--packed", action="store_true", help="accepted for compatibility")
    ap.add_argument("--hierarchical", action="store_true")
    ap.add_argument("--hierarchical-radius", type=int, default=8)  # the runner's default (not the config's 4)
    ap.add_argument("--hierarchical-fallback", default="nearest_valid", choices=sorted(_FB_PARSE))
    ap.add_argument("--hierarchical-no-cross", action="store_true")
    ap.add_argument("--hierarchical-no-fill", action="store_true")
    ap.add_argument("--hierarchical-adaptive", action="store_true")
    ap.add_argument("--hierarchical-confidence-threshold", type=float, default=0.5)
    ap.add_argument("--hierarchical-expanded-radius", type=int, default=8)
    ap.add_argument("--subpixel-method", default="legacy", choices=sorted(_SP_PARSE))
    ap.add_argument("--subpixel-param", type=float, default=None)
    ap.add_argument("--inpaint-method", default="legacy", choices=sorted(_IP_PARSE))
    ap.add_argument("--inpaint-gap", type=lambda v: max(1, int(v)), default=32)
    ap.add_argument("--subpixel-telem", action="store_true")
    ap.add_argument("--inpaint-telem", action="store_true")
    ap.add_argument("--verify-backends", action="store_true", help="not part of the CUDA backend (one layout)")
    args = ap.parse_args(argv)
    if args.subpixel_param is None:  # the method's default parameter (apps/benchmark_stereo.cpp:265-273)
        args.subpixel_param = {1: 4.0, 2: 0.05, 3: 4.0}.get(_SP_PARSE[args.subpixel_method], 0.0)
    if args.verify_backends:
        print("Error: --verify-backends is not part of the CUDA backend", file=sys.stderr)
        return 2
    return run(args)


if __name__ == "__main__":
    sys.exit(main())
