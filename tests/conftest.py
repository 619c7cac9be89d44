"""Test configuration: the `gpu` marker selects tests that need a B200."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 (sm_100a) and the built libfeelmri_b200.so")


@pytest.fixture(scope="session")
def cuda():
    """The CUDA device; GPU tests fail loudly (never skip to a CPU path)."""
    import torch
    assert torch.cuda.is_available(), "gpu-marked test run without a CUDA device"
    return torch.device("cuda", 0)
