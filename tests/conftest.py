import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

import gammcor_pkg  # noqa: E402

gammcor_pkg.load()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long CPU-only oracle runs")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_lib():
    from gammcor_integrals_b200 import _capi
    if not has_gpu():
        pytest.fail("GPU test selected but no CUDA device is visible")
    L = _capi.lib()
    _capi.check(L.gci_init())
    return L
