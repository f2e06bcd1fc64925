import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and liblbm3d.so")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle

    oracle.build()
    oracle.set_threads(min(8, os.cpu_count() or 1))
    return oracle


@pytest.fixture(scope="session")
def gpu():
    """The CUDA device; a GPU test fails (does not skip) when it is absent."""
    import torch

    assert torch.cuda.is_available(), "GPU test run without a CUDA device"
    from lbm3d_bb_b200 import build

    build.build()
    return torch.device("cuda:0")
