import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the native sm_100a library)")
    config.addinivalue_line("markers", "slow: large CPU oracle work")


def cuda_ok() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ctx():
    """One library context for the GPU session (device 0)."""
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import simd_bigint_b200 as sbg
    c = sbg.Context(0)
    yield c
    c.close()
