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


def metric_case(w, h, seed, ch=1, quantised=True, specials=True):
    """Inputs for evaluate_stereo: piecewise-planar GT with steps (disparity boundaries), an
    estimate with small and large errors and invalid pixels, refine maps, visibility with values
    around the 200 threshold, ranges that miss some GT, and a left image with flat and textured
    parts.  quantised: values on grids that keep every double sum exact in any order."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:h, 0:w].astype(np.float32)
    cells = (x // max(4, w // 7)).astype(int) * 7 + (y // max(4, h // 5)).astype(int)
    base = rng.uniform(2, 60, cells.max() + 1).astype(np.float32)
    gt = base[cells] + 0.01 * x - 0.005 * y
    noise = rng.normal(0, 0.6, (h, w)).astype(np.float32)
    big = rng.random((h, w)) < 0.08
    noise[big] += rng.uniform(-12, 12, big.sum()).astype(np.float32)
    if quantised:
        gt = np.round(gt * 256) / 256
        noise = np.round(noise * 65536) / 65536
    gt = gt.astype(np.float32)
    est = (gt + noise).astype(np.float32)
    est[rng.random((h, w)) < 0.06] = -1.0
    before = (gt + noise * 1.5).astype(np.float32)
    after = (gt + noise * 1.1).astype(np.float32)
    if quantised:
        before = (np.round(before.astype(np.float64) * 65536) / 65536).astype(np.float32)
        after = (np.round(after.astype(np.float64) * 65536) / 65536).astype(np.float32)
    after[rng.random((h, w)) < 0.03] = -1.0
    if specials:
        sp = rng.random((h, w))
        gt[sp < 0.02] = np.nan
        gt[(sp >= 0.02) & (sp < 0.03)] = np.inf
        gt[(sp >= 0.03) & (sp < 0.04)] = -2.0
        gt[(sp >= 0.04) & (sp < 0.045)] = 2e5
        est[rng.random((h, w)) < 0.01] = np.nan
        est[rng.random((h, w)) < 0.005] = np.inf
    vis = rng.choice(np.array([0, 150, 199, 200, 201, 255], np.uint8), (h, w), p=[.1, .05, .1, .1, .05, .6])
    g0 = np.nan_to_num(gt, nan=0.0, posinf=0.0, neginf=0.0)
    r = rng.integers(0, 6, (h, w))
    rmin = np.clip(np.floor(g0) - r, -32768, 32767).astype(np.int16)
    rmax = np.clip(np.floor(g0) + r + rng.integers(0, 2, (h, w)), -32768, 32767).astype(np.int16)
    tex = rng.integers(0, 256, (h, w, ch)).astype(np.uint8)
    flat = (x < w // 3)[..., None]
    left = np.where(flat, np.uint8(120), tex).astype(np.uint8)
    if ch == 1:
        left = left[..., 0]
    return {"est": est, "gt": gt, "range": (rmin, rmax), "before": before, "after": after, "vis": vis, "left": left}


def same_metrics(a, b):
    """Field-by-field equality of two StereoMetrics records (floats compared by bit pattern)."""
    import struct
    da, db = a.to_dict(), b.to_dict()

    def flat(d, pre=""):
        for k, v in d.items():
            if isinstance(v, dict):
                yield from flat(v, pre + k + ".")
            else:
                yield pre + k, v

    fa, fb = dict(flat(da)), dict(flat(db))
    bad = []
    for k in fa:
        va, vb = fa[k], fb[k]
        if isinstance(va, float):
            if struct.pack("<f", va) != struct.pack("<f", vb):
                bad.append((k, va, vb))
        elif va != vb:
            bad.append((k, va, vb))
    return bad
