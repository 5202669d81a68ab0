"""The reference's own C-API tests, unchanged, against this library on the GPU.

tests/c_api_smoke.c (pure C99: version, struct_size rejection, BoundedReuse over two frames) and
tests/test_c_api.cpp (lifecycle, error statuses, create_ex, and the C-vs-C++ check at lines 29-94
that compares every output of the C API with the reference's C++ StereoSession bit for bit on a
64x48 pair with stride 80) are compiled from the reference tree by `make -C oracle capi_tests`
into oracle/_ref/.  Every apg_* call in them resolves to apg_sgm_b200/libapg_sgm_b200.so, so the C
side runs the CUDA engine and the C++ side is the reference CPU pipeline.
"""
import subprocess

import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

CASES = [
    ("c_api_smoke", "Pure C API smoke test passed successfully!"),
    ("test_c_api", "All C API tests passed successfully!"),
]


@pytest.mark.parametrize("name,banner", CASES)
def test_reference_c_api_test_passes_unchanged(apg, name, banner):
    exe = O.HERE / "_ref" / name
    if not exe.exists():
        pytest.skip(f"oracle/_ref/{name} not built (make -C oracle capi_tests needs the reference sources)")
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert banner in r.stdout
