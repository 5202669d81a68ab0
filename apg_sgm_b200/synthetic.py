"""Seeded synthetic rectified stereo pairs.

These stand in for the public KITTI 2012/2015 and Middlebury 2014 scenes the reference
benchmarks on (its manifests under benchmarks/manifests/), which are not available here.  The
recipe, per pair:

1. Left image: uniform noise, Gaussian blur (sigma 1.5 px), rescaled to 0..255, with
   constant-intensity patches (two 60x60 patches, or about 20 % of the area for the
   1920x1080 HighQuality workload).
2. Ground truth: a Voronoi partition of K seeded points; every cell is a plane
   d = a + b*x + c*y with b, c in [-0.02, 0.02] and d clipped to [d_lo, d_hi].
3. Right image: forward warp right(x - round(d), y) = left(x, y); where two pixels land on
   the same target the larger disparity wins; target pixels nobody lands on get fresh noise
   (occlusions).
4. Additive Gaussian noise (sigma 2) on both images, clamped to uint8.

Pair i of a workload uses seed 0xA9650000 + i.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

SEED_BASE = 0xA9650000


@dataclass(frozen=True)
class PairSpec:
    width: int
    height: int
    max_disparity: int
    cells: int
    d_lo: int
    d_hi: int
    patch_fraction: float = 0.0  # 0 -> two 60x60 patches


# The workloads named by the benchmark configuration (shape, disparity range, Voronoi cells).
BALANCED_640 = PairSpec(640, 480, 64, 8, 4, 60)
FAST_720P = PairSpec(1280, 720, 128, 12, 0, 120)
HQ_1080P = PairSpec(1920, 1080, 256, 16, 0, 240, patch_fraction=0.2)
KITTI_1242 = PairSpec(1242, 375, 192, 12, 0, 180)


def _blur(img: np.ndarray, sigma: float) -> np.ndarray:
    r = int(np.ceil(3 * sigma))
    k = np.exp(-0.5 * (np.arange(-r, r + 1) / sigma) ** 2)
    k /= k.sum()
    p = np.pad(img, r, mode="reflect")
    tmp = np.zeros((p.shape[0], img.shape[1]), np.float64)
    for i, kv in enumerate(k):
        tmp += kv * p[:, i:i + img.shape[1]]
    out = np.zeros(img.shape, np.float64)
    for i, kv in enumerate(k):
        out += kv * tmp[i:i + img.shape[0], :]
    return out


def make_pair(spec: PairSpec, seed: int):
    """(left u8 HxW, right u8 HxW, ground-truth disparity f32 HxW)."""
    rng = np.random.default_rng(seed)
    w, h = spec.width, spec.height
    base = _blur(rng.random((h, w)), 1.5)
    base = (base - base.min()) / max(base.max() - base.min(), 1e-9) * 255.0
    left = base.copy()
    if spec.patch_fraction <= 0.0:
        for _ in range(2):
            ps = min(60, w, h)
            x0 = int(rng.integers(0, max(1, w - ps + 1)))
            y0 = int(rng.integers(0, max(1, h - ps + 1)))
            left[y0:y0 + ps, x0:x0 + ps] = float(rng.integers(0, 256))
    else:
        target = spec.patch_fraction * w * h
        covered = np.zeros((h, w), bool)
        while covered.sum() < target:
            pw = int(rng.integers(40, 160)); ph = int(rng.integers(40, 160))
            x0 = int(rng.integers(0, max(1, w - pw))); y0 = int(rng.integers(0, max(1, h - ph)))
            left[y0:y0 + ph, x0:x0 + pw] = float(rng.integers(0, 256))
            covered[y0:y0 + ph, x0:x0 + pw] = True

    # Ground truth: Voronoi cells, each a clipped plane.
    k = spec.cells
    sx = rng.uniform(0, w, k); sy = rng.uniform(0, h, k)
    a = rng.uniform(spec.d_lo, spec.d_hi, k)
    b = rng.uniform(-0.02, 0.02, k); c = rng.uniform(-0.02, 0.02, k)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    best = np.full((h, w), np.inf); label = np.zeros((h, w), np.int64)
    for i in range(k):
        dist = (xx - sx[i]) ** 2 + (yy - sy[i]) ** 2
        m = dist < best
        best[m] = dist[m]; label[m] = i
    gt = a[label] + b[label] * (xx - sx[label]) + c[label] * (yy - sy[label])
    gt = np.clip(gt, spec.d_lo, spec.d_hi)

    # Forward warp, larger disparity wins.
    di = np.rint(gt).astype(np.int64)
    xt = xx.astype(np.int64) - di
    ok = (xt >= 0) & (xt < w)
    right = rng.random((h, w)) * 255.0
    zbuf = np.full((h, w), -1, np.int64)
    ys, xs = np.nonzero(ok)
    np.maximum.at(zbuf, (ys, xt[ys, xs]), di[ys, xs])
    win = di[ys, xs] == zbuf[ys, xt[ys, xs]]  # one source per target: same d -> distinct x
    right[ys[win], xt[ys[win], xs[win]]] = left[ys[win], xs[win]]

    left = left + rng.normal(0.0, 2.0, (h, w))
    right = right + rng.normal(0.0, 2.0, (h, w))
    L = np.clip(np.rint(left), 0, 255).astype(np.uint8)
    R = np.clip(np.rint(right), 0, 255).astype(np.uint8)
    return L, R, gt.astype(np.float32)


def pair_for(spec: PairSpec, index: int = 0):
    return make_pair(spec, SEED_BASE + index)


def batched_mix():
    """The 64-pair uneven batch: 24 x 640x480 D64, 24 x 1242x375 D192, 16 x 1280x720 D128
    (4,505,472,000 voxels), pair i seeded SEED_BASE + i."""
    specs = [BALANCED_640] * 24 + [KITTI_1242] * 24 + [FAST_720P] * 16
    return specs
