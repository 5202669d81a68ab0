"""Generate tests/golden/hier_fixtures.npz from the REFERENCE implementation.

Runs the reference's hierarchical coarse-to-fine search range
(HierarchicalStereo::estimate_search_range) and its full pipeline in hierarchical mode
(oracle/_ref/libapg_ref.so, compiled from the reference sources by oracle/Makefile, entry
ref_hier_dump of oracle/ref_shim.cpp) on small seeded inputs, and stores inputs, configurations,
the range planes, the guiding disparity, the telemetry and the final maps.  The committed
fixtures pin the C oracle's restatement where the reference tree is not available.

    make -C oracle ref && python tests/golden/make_golden_hier.py
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

OUT = Path(__file__).resolve().parent / "hier_fixtures.npz"

CASES = [
    # name, mode, dmax, dmin, (inputs, w, h, seed), hierarchical overrides
    ("balanced_128x96_d32", 1, 32, 0, ("synth_patch", 128, 96, 1), {}),
    ("fast_96x64_d32", 0, 32, 0, ("synth", 96, 64, 2), {}),
    ("adaptive_101x67_d48", 1, 48, 0, ("synth_patch", 101, 67, 3), {"hier_adaptive_radius": 1}),
    ("fullrange_nofill_80x60_d40", 1, 40, 4, ("synth_patch", 80, 60, 4),
     {"hier_fallback": 1, "hier_coarse_fill_holes": 0}),
    ("expanded_nocross_80x60_d40", 1, 40, 0, ("synth_patch", 80, 60, 5),
     {"hier_fallback": 2, "hier_coarse_cross_agg": 0, "hier_radius": 3}),
    ("nearest_nofill_96x72_d48", 1, 48, 6, ("synth_patch", 96, 72, 6), {"hier_coarse_fill_holes": 0}),
    ("hq_96x64_d32", 2, 32, 0, ("synth_patch", 96, 64, 7), {}),
    ("negative_72x48", 1, 24, -8, ("synth", 72, 48, 8), {}),
    ("rgb_64x48_d16", 1, 16, 0, ("rgb_shift", 64, 48, 0), {}),
    ("small_40x20_d16", 1, 16, 0, ("synth", 40, 20, 9), {}),
]

KEYS = ["range_min", "range_max", "d_prior", "disparity", "confidence", "invalid_reason", "reliable_mask"]


def make_inputs(kind, w, h, seed, dmax):
    if kind == "synth":
        return synth(w, h, dmax, cells=5, lo=0, hi=dmax * 3 // 4, seed=seed)
    if kind == "synth_patch":
        return synth(w, h, dmax, cells=5, lo=0, hi=dmax * 3 // 4, patch=0.2, seed=seed)
    left = pattern(w, h, 3, "noise")
    return left, np.roll(left, -3, axis=1)


def main():
    if not O.ref_available():
        raise SystemExit("build the reference first: make -C oracle ref")
    data, names = {}, []
    for name, mode, dmax, dmin, (kind, w, h, seed), over in CASES:
        cfg = O.config(mode, dmax, dmin, hier_enable=1, **over)
        L, R = make_inputs(kind, w, h, seed, dmax)
        d = O.ref_hier_dump(cfg, L, R)
        assert d["status"] == 0, (name, d["status"])
        names.append(name)
        data[f"{name}/left"] = L
        data[f"{name}/right"] = R
        data[f"{name}/config"] = np.frombuffer(bytes(cfg), np.uint8)
        for k in KEYS:
            data[f"{name}/{k}"] = d[k]
        t = d["telemetry"]
        data[f"{name}/telemetry"] = np.array([t["avg_states_per_pixel"], t["coarse_valid_ratio"],
                                              t["fallback_pixel_ratio"], t["full_range_pixel_ratio"], d["ran"]])
    data["cases"] = np.array(names)
    np.savez_compressed(OUT, **data)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes, {len(names)} cases)")


if __name__ == "__main__":
    main()
