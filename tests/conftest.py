import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def _ensure_oracle():
    so = ROOT / "oracle" / "liboracle.so"
    if not so.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "oracle"], check=True, capture_output=True)


@pytest.fixture(scope="session")
def O():
    _ensure_oracle()
    from oracle import oracle as mod
    return mod


@pytest.fixture(scope="session")
def apg():
    import apg_sgm_b200 as mod
    return mod
