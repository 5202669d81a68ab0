"""Generate tests/golden/metrics_fixtures.npz from the REFERENCE implementation.

Runs the reference's evaluate_stereo (src/metrics.cpp, compiled from the reference sources by
oracle/Makefile into oracle/_ref/libapg_ref.so; entry ref_evaluate_stereo of oracle/ref_shim.cpp)
on the seeded inputs of tests/test_metrics.py's cases (tests/helpers.py metric_case) and stores
each result record (apg_stereo_metrics_t bytes).  The inputs are regenerated from their seeds.

    make -C oracle ref && python tests/golden/make_golden_metrics.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

from oracle import oracle as O  # noqa: E402
from test_metrics import CASES, run_case  # noqa: E402

OUT = Path(__file__).resolve().parent / "metrics_fixtures.npz"


def main():
    if not O.ref_available():
        raise SystemExit("build the reference first: make -C oracle ref")
    data, names = {}, []
    for case in CASES:
        rec = run_case(lambda *a: O.evaluate_stereo(*a, reference=True), case)
        data[f"{case[0]}/record"] = np.frombuffer(bytes(rec), np.uint8)
        names.append(case[0])
    data["cases"] = np.array(names)
    np.savez_compressed(OUT, **data)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes, {len(names)} cases)")


if __name__ == "__main__":
    main()
