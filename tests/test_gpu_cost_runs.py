"""The pixel-run cost kernel against the column-tile kernel: same volumes, same argmin, same maps.

The run form (cost_runs.cu) is the default for the 32-bit census with default ranges; the tuning
key cost_kernel=1 forces the tile form (cost.cu).  Both must give bit-identical raw volumes, cross-H
aggregated volumes, right-image disparities and final maps over the shapes that exercise the
run kernel's edges: odd and padded disparity counts, negative minimum disparity, images narrower
than a tile or than the disparity range, the three-warp word sets of D=192, D=256, the cost
forms (census only, AD only, gradient only, all three; with and without aggregation) and the
per-pixel ranges of the HighQuality prior.  The
stage-parity tests check the same kernels against the oracle.
"""
import zlib

import pytest

from helpers import same_bits, synth

pytestmark = pytest.mark.gpu

DUMPS = ("cost_raw", "cost_agg", "disp_right")

CASES = [
    # name, mode, w, h, dmax, dmin, overrides
    ("balanced_300x90_d96", 1, 300, 90, 96, 0, {}),
    ("balanced_1280x24_d128", 1, 1280, 24, 128, 0, {}),
    ("balanced_odd_d99", 1, 200, 40, 99, 0, {}),
    ("balanced_neg_dmin", 1, 160, 48, 40, -24, {}),
    ("balanced_d192", 1, 420, 30, 192, 0, {}),
    ("balanced_d256", 1, 333, 20, 256, 0, {}),
    ("balanced_narrow_20", 1, 20, 70, 64, 0, {}),
    ("balanced_narrow_70x33", 1, 70, 33, 128, 0, {}),
    ("balanced_arm5", 1, 256, 40, 64, 0, {"max_arm_length": 5}),
    ("balanced_ad_only", 1, 200, 40, 64, 0, {"use_grad": False}),
    ("balanced_grad_only", 1, 200, 40, 64, 0, {"use_ad": False}),
    ("census_agg", 1, 200, 40, 64, 0, {"use_ad": False, "use_grad": False}),
    ("fast_300x90_d96", 0, 300, 90, 96, 0, {}),
    ("fast_odd_d65", 0, 513, 31, 65, 0, {}),
    ("fast_neg_dmin", 0, 130, 30, 32, -32, {}),
    ("fast_full_costs", 0, 200, 40, 64, 0, {"use_ad": True, "use_grad": True}),
    # per-pixel ranges from the prior (HighQuality): range masks per voxel, count prefixes
    ("hq_300x90_d96", 2, 300, 90, 96, 0, {}),
    ("hq_333x40_d256", 2, 333, 40, 256, 0, {}),
    ("hq_neg_dmin", 2, 160, 48, 40, -24, {}),
    ("hq_narrow_70x33", 2, 70, 33, 128, 0, {}),
    ("hq_census_agg", 2, 200, 60, 64, 0, {"use_ad": False, "use_grad": False}),
]


def _run(apg, cfg, L, R, kernel, fused=False, debug=True):
    e = apg.Engine(cfg, debug=(apg.DEBUG_RAW_COST if debug else 0))
    e.set_tuning("cost_kernel", kernel)
    if fused:
        e.set_tuning("fast_fused", 1)
    out = e.process(L, R)
    # the aggregated volume exists only with aggregation on
    names = [k for k in DUMPS if k != "cost_agg" or cfg.agg_enable]
    dumps = {k: e.dump(k) for k in names} if debug else {}
    e.close()
    return out, dumps


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_runs_equal_tiles(apg, case):
    name, mode, w, h, dmax, dmin, over = case
    cfg = apg.config_from_mode(mode, dmax, dmin, **over)
    L, R = synth(w, h, max(dmax, 8), patch=0.2 if mode == 2 else 0.0, seed=zlib.crc32(name.encode()) % 1000)
    a, da = _run(apg, cfg, L, R, 0)
    b, db = _run(apg, cfg, L, R, 1)
    for k in a:
        assert same_bits(a[k], b[k]), (name, k)
    assert da.keys() == db.keys()
    for k in da:
        assert same_bits(da[k], db[k]), (name, k)


@pytest.mark.parametrize("w,h,dmax", [(300, 90, 96), (1280, 16, 128), (70, 33, 64)])
def test_runs_fused_fast_equal_tiles(apg, w, h, dmax):
    """The fused Fast form (no volume stored, right-image argmin only) gives the same maps."""
    cfg = apg.config_from_mode(0, dmax)
    L, R = synth(w, h, dmax, seed=5)
    a, _ = _run(apg, cfg, L, R, 0, fused=True, debug=False)
    b, _ = _run(apg, cfg, L, R, 1, fused=True, debug=False)
    c, _ = _run(apg, cfg, L, R, 1, fused=False, debug=False)
    for k in a:
        assert same_bits(a[k], b[k]), k
        assert same_bits(a[k], c[k]), k


def test_cost_kernel_key_rejects_unknown(apg):
    e = apg.Engine(apg.config_from_mode(1, 64))
    with pytest.raises(Exception):
        e.set_tuning("cost_kernel", 2)
    e.close()
