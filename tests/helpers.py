"""Shared helpers for the parity tests (inputs, config conversion, comparisons)."""
import numpy as np

from apg_sgm_b200 import synthetic as S


def to_oracle(O, cfg):
    """Copy a product apg_pipeline_config_t into the oracle's identical ctypes struct."""
    return O.PipelineConfig.from_buffer_copy(bytes(cfg))


def pattern(w, h, ch, kind):
    """The reference contract patterns (tests/test_api_contract.cpp:43-74)."""
    yy, xx = np.mgrid[0:h, 0:w]
    if kind == "checker":
        v = np.where(((xx // 4 + yy // 4) % 2) == 0, 40, 210)
    elif kind == "noise":
        v = (xx * 37 + yy * 73 + xx * yy * 13) % 256
    elif kind == "hramp":
        v = (xx * 255) // max(1, w - 1)
    elif kind == "vramp":
        v = (yy * 255) // max(1, h - 1)
    else:
        v = np.full((h, w), 128)
    v = v.astype(np.uint8)
    if ch == 1:
        return v
    return np.stack([v, (v.astype(int) + 30) % 256, (v.astype(int) + 60) % 256], -1).astype(np.uint8)


def synth(w, h, dmax, cells=6, lo=0, hi=None, patch=0.0, seed=0):
    spec = S.PairSpec(w, h, dmax, cells, lo, hi if hi is not None else max(lo, dmax - 4), patch)
    L, R, _ = S.make_pair(spec, S.SEED_BASE + seed)
    return L, R


def same_bits(a, b):
    a = np.ascontiguousarray(a); b = np.ascontiguousarray(b)
    return a.shape == b.shape and a.dtype == b.dtype and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def diff_report(a, b):
    a = np.asarray(a); b = np.asarray(b)
    if a.shape != b.shape:
        return f"shape {a.shape} vs {b.shape}"
    bad = np.argwhere(a.view(np.uint8).reshape(a.shape + (-1,)).any(-1) if False else (a != b))
    n = int((a != b).sum())
    first = tuple(int(i) for i in bad[0]) if len(bad) else None
    return f"{n} mismatches; first at {first}: {a[first] if first else None} vs {b[first] if first else None}"
