"""The manifest benchmark runner against the reference's own runner (apps/benchmark_stereo.cpp,
built from the reference sources into oracle/_ref/benchmark_stereo) on the same manifest: every
CSV column except those that measure this machine (times, bytes, thread counts, backend name) must
be identical."""
import csv
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SKIP = {"backend", "threads", "effective_threads", "cost_bytes", "cost32_bytes", "peak_bytes",
        "peak_workspace_bytes", "retained_workspace_bytes"}


def _manifest(apg, d):
    from apg_sgm_b200 import synthetic as S
    lines = ["# synthetic cases", ""]
    for i, (w, h, D) in enumerate([(160, 96, 32), (128, 80, 48)]):
        L, R, gt = S.make_pair(S.PairSpec(w, h, D, 6, 0, D * 3 // 4, 0.1), 100 + i)
        gt = (np.round(gt.astype(np.float64) * 256) / 256).astype(np.float32)
        apg.save_pgm(d / f"l{i}.pgm", L)
        apg.save_pgm(d / f"r{i}.pgm", R)
        apg.save_pfm(d / f"gt{i}.pfm", gt)
        vis = np.where(np.arange(w)[None, :] - np.round(gt) >= 0, 255, 0).astype(np.uint8)
        apg.save_pgm(d / f"v{i}.pgm", vis)
        lines.append(f"case{i} l{i}.pgm r{i}.pgm gt{i}.pfm {D} 0 v{i}.pgm" if i == 0 else
                     f"case{i} l{i}.pgm r{i}.pgm gt{i}.pfm {D}")
    lines.append("nogt l0.pgm r0.pgm missing.pfm 32")
    (d / "m.txt").write_text("\n".join(lines) + "\n")
    return d / "m.txt"


@pytest.mark.parametrize("extra", [[], ["--subpixel-method", "conf_gate", "--inpaint-method", "shadow_reclass",
                                        "--inpaint-gap", "12"],
                                   ["--hierarchical", "--hierarchical-adaptive", "--hierarchical-fallback", "expanded"],
                                   ["--subpixel-method", "stabilized", "--subpixel-telem", "--inpaint-telem",
                                    "--repeat", "2"]],
                         ids=["default", "scopes", "hierarchical", "telemetry"])
def test_runner_matches_reference_runner(O, apg, tmp_path, extra):
    exe = O.HERE / "_ref" / "benchmark_stereo"
    if not exe.exists():
        pytest.skip("reference runner (oracle/_ref/benchmark_stereo) not built")
    from apg_sgm_b200 import benchmark as B
    m = _manifest(apg, tmp_path)
    args = ["--manifest", str(m), "--ablation", "A,C,E,F", "--warmup", "0"] + \
        (["--repeat", "1"] if "--repeat" not in extra else []) + extra
    r = subprocess.run([str(exe)] + args + ["--output", str(tmp_path / "ref.csv")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert B.main(args + ["--output", str(tmp_path / "ours.csv")]) == 0
    ref = list(csv.DictReader(open(tmp_path / "ref.csv")))
    ours = list(csv.DictReader(open(tmp_path / "ours.csv")))
    assert len(ref) == len(ours) == 12
    for a, b in zip(ref, ours):
        for k in a:
            if k in SKIP or k.startswith("time_"):
                continue
            assert a[k] == b[k], (a["case"], a["ablation_id"], k, a[k], b[k])
