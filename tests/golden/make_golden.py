"""Generate tests/golden/reference_fixtures.npz from the REFERENCE implementation.

Runs the reference's own pipeline (oracle/_ref/libapg_ref.so, compiled from the reference
sources by oracle/Makefile) on small seeded inputs and stores inputs, configurations and the
reference's outputs (final maps plus the WTA / right-WTA / confidence stages, and the cost
volumes of the smallest case).  The committed fixtures pin the C oracle where the reference
tree is not available.

    make -C oracle ref && python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

from oracle import oracle as O  # noqa: E402
from helpers import pattern, synth  # noqa: E402

OUT = Path(__file__).resolve().parent / "reference_fixtures.npz"

CASES = [
    # name, mode, dmax, dmin, inputs, overrides, keep volumes
    ("fast_64x48_d16", 0, 16, 0, ("synth", 64, 48, 0), {}, False),
    ("balanced_64x48_d16", 1, 16, 0, ("synth", 64, 48, 1), {}, False),
    ("balanced_33x27_d16_checker", 1, 16, 0, ("checker_shift", 33, 27, 0), {}, True),
    ("hq_160x120_d32", 2, 32, 0, ("synth_patch", 160, 120, 2), {}, False),
    ("negative_48x36", 1, 8, -4, ("noise_shift", 48, 36, 0), {}, False),
    ("rgb_balanced_32x24", 1, 16, 0, ("rgb_shift", 32, 24, 0), {}, False),
    ("census9x7_balanced_64x48", 1, 24, 0, ("synth", 64, 48, 3), {"census_type": 0}, False),
    ("path8_balanced_80x60", 1, 24, 0, ("synth", 80, 60, 4), {"paths": 8}, False),
]

STAGES = ["disp_wta", "best", "second", "disp_right", "conf_confidence", "conf_reliable", "conf_reason",
          "disp_refined", "disp_lr", "reason_lr", "disp_fill", "disparity", "confidence", "invalid_reason",
          "reliable_mask", "range_min", "range_max", "d_prior"]


def make_inputs(kind, w, h, seed, dmax):
    if kind == "synth":
        return synth(w, h, dmax, cells=5, lo=0, hi=dmax * 3 // 4, seed=seed)
    if kind == "synth_patch":
        return synth(w, h, dmax, cells=5, lo=0, hi=dmax * 3 // 4, patch=0.2, seed=seed)
    base = {"checker_shift": ("checker", 1), "noise_shift": ("noise", 1), "rgb_shift": ("noise", 3)}[kind]
    left = pattern(w, h, base[1], base[0])
    return left, np.roll(left, -3, axis=1)


def main():
    if not O.ref_available():
        raise SystemExit("build the reference first: make -C oracle ref")
    data = {}
    names = []
    for name, mode, dmax, dmin, (kind, w, h, seed), over, vols in CASES:
        cfg = O.config(mode, dmax, dmin, **over)
        L, R = make_inputs(kind, w, h, seed, dmax)
        d = O.ref_dump(cfg, L, R)
        assert d["status"] == 0, (name, d["status"])
        names.append(name)
        data[f"{name}/left"] = L
        data[f"{name}/right"] = R
        data[f"{name}/config"] = np.frombuffer(bytes(cfg), np.uint8)
        data[f"{name}/support_count"] = np.array(d["support_count"])
        for s in STAGES:
            data[f"{name}/{s}"] = d[s]
        if vols:
            data[f"{name}/cost_raw"] = d["cost_raw"]
            data[f"{name}/cost_agg"] = d["cost_agg"]
            data[f"{name}/sgm_sum"] = d["sgm_sum"]
    data["cases"] = np.array(names)
    np.savez_compressed(OUT, **data)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes, {len(names)} cases)")


if __name__ == "__main__":
    main()
