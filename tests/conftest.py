import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a kernels)")
    config.addinivalue_line("markers", "slow: long statistical runs")


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    """Skips a GPU test when no device is present (CPU-only runs)."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    import torch

    torch.cuda.init()
    return torch


@pytest.fixture(scope="session")
def engine_lib():
    from dsmc_erlend_b200 import _lib
    from dsmc_erlend_b200.build import build

    if not _lib.LIB_PATH.exists():
        build()
    return _lib.load()
