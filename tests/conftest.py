import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device; runs the sm_100a kernels")


@pytest.fixture(scope="session")
def lib():
    """The built libtcb200.so (built in-tree first if it is missing or stale)."""
    from torchcor_b200 import build as b
    from torchcor_b200 import _lib
    b.build()
    return _lib.load()


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    return torch.device("cuda:0")
