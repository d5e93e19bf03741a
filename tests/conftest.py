import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")
    config.addinivalue_line("markers", "slow: long CPU-oracle run")


@pytest.fixture(scope="session")
def golden():
    return GOLDEN


def cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
