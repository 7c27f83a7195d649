import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")
    config.addinivalue_line("markers", "slow: long-running (large sizes)")


@pytest.fixture(scope="session")
def uw12lib():
    """The built CUDA library (rebuilt in-tree when a source is newer)."""
    import libuw12_b200
    from libuw12_b200 import build
    build.build()
    return libuw12_b200


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("no CUDA device: GPU tests must run on a B200")
    torch.cuda.init()
    return torch.device("cuda:0")
