import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (run with -m gpu)")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the product and the oracle once per session (incremental)."""
    from lmie_b200 import build
    build.build()
    import subprocess
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)
    yield
