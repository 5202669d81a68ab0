"""Host-side logic and the C-ABI boundary, on the CPU (no GPU needed)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _has_cuda_device():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_division_magic_is_exact():
    """Every (n, d) the cross aggregation divides: n < 2^16 window sums, 1 <= d <= 255 counts."""
    n = np.arange(1 << 16, dtype=np.uint64)
    for d in range(2, 256):
        m = np.uint64((1 << 32) // d + 1)
        q = (n * m) >> np.uint64(32)
        assert np.array_equal(q, n // np.uint64(d)), d


def _declared(header: Path, macro: str):
    """Function names of `MACRO <return type> name(` declarations (not the #define line)."""
    text = header.read_text()
    return re.findall(rf"^\s*{macro}\s+(?:const\s+)?\w+[\s\*]+(\w+)\s*\(", text, flags=re.MULTILINE)


def test_library_exports_every_declared_symbol():
    from apg_sgm_b200 import _lib
    lib = _lib.lib()
    names = _declared(ROOT / "include" / "apg_sgm" / "c_api.h", "APG_API") + \
        _declared(ROOT / "include" / "apg_sgm_cuda.h", "APGCU_API")
    assert len(names) > 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding declares a signature for each of them
    assert set(names) <= set(_lib.declared_symbols()), set(names) - set(_lib.declared_symbols())


def test_abi_struct_layouts_match_headers(tmp_path):
    """Compile the public headers with gcc and compare sizes/offsets with the ctypes mirrors."""
    from apg_sgm_b200 import _lib
    src = tmp_path / "layout.c"
    fields = [f for f, _ in _lib.PipelineConfig._fields_]
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "apg_sgm_cuda.h"', "int main(void) {",
             'printf("%zu %zu %zu\\n", sizeof(apg_pipeline_config_t), sizeof(apg_session_options_t), '
             'sizeof(apg_image_view_t));',
             'printf("%zu %zu\\n", offsetof(apg_session_options_t, max_retained_bytes), '
             'offsetof(apg_session_options_t, max_disparity));']
    for f in fields:
        lines.append(f'printf("%zu\\n", offsetof(apg_pipeline_config_t, {f}));')
    lines.append("return 0; }")
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    vals = [int(v) for v in out]
    assert vals[0] == C.sizeof(_lib.PipelineConfig)
    assert vals[1] == C.sizeof(_lib.SessionOptions)
    assert vals[2] == C.sizeof(_lib.ImageView)
    assert vals[3] == _lib.SessionOptions.max_retained_bytes.offset
    assert vals[4] == _lib.SessionOptions.max_disparity.offset
    for f, off in zip(fields, vals[5:]):
        assert getattr(_lib.PipelineConfig, f).offset == off, f


def test_config_from_mode_matches_reference_presets(O):
    """apgcu_config_from_mode == the oracle's restatement of PipelineConfig::from_mode."""
    import apg_sgm_b200 as apg
    for mode in (0, 1, 2):
        for dmax in (16, 64, 128, 256):
            a = apg.config_from_mode(mode, dmax)
            b = O.config(mode, dmax)
            a.volume_backend = b.volume_backend
            assert bytes(a) == bytes(b), (mode, dmax)


def _session(lib, mode=1, policy=0, budget=0, dmin=0, dmax=64, size=None):
    from apg_sgm_b200 import _lib
    o = _lib.SessionOptions()
    o.struct_size = C.sizeof(_lib.SessionOptions) if size is None else size
    o.quality_mode, o.memory_policy, o.max_retained_bytes = mode, policy, budget
    o.min_disparity, o.max_disparity, o.backend = dmin, dmax, 3
    return lib.apg_session_create_ex(C.byref(o))


def _view(a, stride=None, ch=1):
    from apg_sgm_b200 import _lib
    h, w = a.shape[:2]
    return _lib.ImageView(a.ctypes.data, w, h, stride if stride is not None else a.strides[0], ch)


def test_c_api_contract_on_host():
    """Boundary semantics that need no GPU (src/c_api.cpp:10-204, tests/test_hardening.cpp)."""
    from apg_sgm_b200 import _lib
    L = _lib.lib()
    assert L.apg_version_string() == b"1.0.0"
    assert L.apg_status_string(0) == b"Ok"
    assert L.apg_status_string(6) == b"ResourceLimitExceeded"
    assert L.apg_status_string(99) == b"Unknown"
    # struct_size must be 0 or sizeof
    assert not _session(L, size=12)
    assert _session(L, size=0)
    s = _session(L)
    r = L.apg_result_create()
    img = np.zeros((48, 64), np.uint8)
    # null handles / pointers
    assert L.apg_session_process(None, None, None, r) == 8
    assert L.apg_session_process(s, None, C.byref(_view(img)), r) == 1
    assert L.apg_session_get_last_error(s) == b"Null input pointer"
    # stride smaller than the row
    assert L.apg_session_process(s, C.byref(_view(img, 16)), C.byref(_view(img, 16)), r) == 2
    # size mismatch
    other = np.zeros((48, 60), np.uint8)
    assert L.apg_session_process(s, C.byref(_view(img)), C.byref(_view(other)), r) == 2
    assert L.apg_session_get_frame_count(s) == 0
    w, h = C.c_int(-1), C.c_int(-1)
    assert not L.apg_result_get_disparity(r, C.byref(w), C.byref(h)) and w.value == 0 and h.value == 0
    # the budget gate rejects before allocating anything (tests/test_hardening.cpp:41-62)
    g = _session(L, mode=0, budget=10 * 1024)
    big = np.full((240, 320), 128, np.uint8)
    assert L.apg_session_process(g, C.byref(_view(big)), C.byref(_view(big)), r) == 6
    assert L.apg_session_get_allocated_bytes(g) == 0
    assert b"budget" in L.apg_session_get_last_error(g)
    # invalid disparity range through the configuration-level constructor
    import apg_sgm_b200 as apg
    cfg = apg.config_from_mode(1, 32)
    cfg.min_disparity = 64
    bad = L.apgcu_session_create_config(C.byref(cfg), 0, 0)
    assert L.apg_session_process(bad, C.byref(_view(img)), C.byref(_view(img)), r) == 3
    for h_ in (s, g, bad):
        L.apg_session_destroy(h_)
    L.apg_result_destroy(r)
    L.apg_session_destroy(None)  # no-ops on NULL
    L.apg_result_destroy(None)


@pytest.mark.skipif(_has_cuda_device(), reason="checks the no-device error path")
def test_no_device_fails_loudly():
    import apg_sgm_b200 as apg
    s = apg.StereoSession(mode="fast", max_disparity=16)
    img = np.zeros((48, 64), np.uint8)
    with pytest.raises(RuntimeError, match=r"\[5\].*CUDA"):
        s.process(img, img)


def test_python_api_errors():
    import apg_sgm_b200 as apg
    with pytest.raises(ValueError, match="Unrecognized mode"):
        apg.StereoSession(mode="super_fast")
    with pytest.raises(ValueError, match="Unrecognized backend"):
        apg.StereoSession(backend="quantum")
    with pytest.raises(ValueError, match="Unrecognized memory_policy"):
        apg.StereoSession(memory_policy="infinite_cache")
    with pytest.raises(RuntimeError, match="strictly greater"):
        apg.StereoSession(min_disparity=64, max_disparity=32)
    s = apg.StereoSession(mode="fast", max_disparity=16)
    assert s.frame_count == 0 and s.total_time_ms == 0.0 and s.allocated_bytes == 0
    assert "StereoSession" in repr(s)
    img = np.zeros((48, 64), np.uint8)
    with pytest.raises(TypeError, match="uint8"):
        s.process(img.astype(np.float32), img)
    with pytest.raises(ValueError, match="2D"):
        s.process(np.zeros((4,), np.uint8), img)
    with pytest.raises(ValueError, match="1 or 3 channels"):
        s.process(np.zeros((48, 64, 2), np.uint8), np.zeros((48, 64, 2), np.uint8))
    with pytest.raises(ValueError, match="identical dimensions"):
        s.process(img, np.zeros((48, 63), np.uint8))
    with pytest.raises(ValueError, match="matching channel"):
        s.process(img, np.zeros((48, 64, 3), np.uint8))
    assert apg.QualityMode.HighQuality == 2 and apg.MemoryPolicy.BoundedReuse == 1
    assert apg.StatusCode.AllocationFailure == 7


def test_workspace_estimates():
    import apg_sgm_b200 as apg
    fast = apg.config_from_mode(0, 128)
    bal = apg.config_from_mode(1, 128)
    wf = apg.workspace_bytes(fast, 1280, 720)
    wb = apg.workspace_bytes(bal, 1280, 720)
    vol = 1280 * 720 * 128 * 2
    assert 4 * vol <= wf < 5 * vol      # Fast: the census cost volume and three first-phase path sums
    assert 4 * vol <= wb < 5 * vol      # Balanced: cross tmp (= first sum buffer), aggregated cost, 2 more sums
    assert apg.workspace_bytes(fast, 640, 480) < wf
    # Fast at a padded range of 256: the census cost volume at one byte per voxel
    w256 = apg.workspace_bytes(apg.config_from_mode(0, 256), 1920, 1080)
    vol256 = 1920 * 1080 * 256 * 2
    assert 3.5 * vol256 <= w256 < 4.5 * vol256


def test_synthetic_generator_is_deterministic():
    from apg_sgm_b200 import synthetic as S
    a = S.make_pair(S.BALANCED_640, S.SEED_BASE)
    b = S.make_pair(S.BALANCED_640, S.SEED_BASE)
    c = S.make_pair(S.BALANCED_640, S.SEED_BASE + 1)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert not np.array_equal(a[0], c[0])
    L, R, gt = a
    assert L.shape == (480, 640) and L.dtype == np.uint8 and R.dtype == np.uint8
    assert gt.min() >= 4 and gt.max() <= 60
    specs = S.batched_mix()
    assert len(specs) == 64
    assert sum(s.width * s.height * s.max_disparity for s in specs) == 4_505_472_000


def test_result_pool_lends_and_takes_back(apg):
    """StereoSession's result pool: a result lent to live arrays is not lent again; it comes back
    when the last array viewing it is gone; beyond `keep` idle results the rest are destroyed."""
    from apg_sgm_b200 import _ResultLease, _ResultPool

    pool = _ResultPool(keep=2)
    a = pool.take()
    b = pool.take()
    assert a and b and a != b
    la, lb = _ResultLease(pool, a), _ResultLease(pool, b)
    holder = [la]
    del la
    assert pool._free == []          # still held
    holder.clear()
    assert pool._free == [a]         # back once nothing holds it
    del lb
    assert sorted(pool._free) == sorted([a, b])
    c = pool.take()
    assert c in (a, b)
    extra = [pool.take() for _ in range(3)]
    for r in extra + [c]:
        pool.give_back(r)
    assert len(pool._free) == 2      # the rest were destroyed
    pool.close()
    assert pool._free == []
