import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _build_once():
    # Build the oracle (CPU) and the CUDA library when they are missing or
    # stale; nvcc cross-compiles without a GPU.
    from oracle import build as ob
    ob.build()
    from cup2d_b200 import build as cb
    cb.build()


_build_once()


@pytest.fixture(scope="session")
def has_gpu():
    import torch
    return torch.cuda.is_available()


@pytest.fixture
def cuda(has_gpu):
    if not has_gpu:
        pytest.fail("GPU test run without a CUDA device")
    import torch
    return torch.device("cuda:0")
