import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA path")


@pytest.fixture(scope="session")
def small_geo():
    """A small helical scan: 96 cols x 8 rows, 120 views/rot, 2 blocks of 32 slices, 32^2."""
    from listctrecons_b200.scan import ScanGeometry

    g = ScanGeometry(ns=96, nt=8, ds=1.0, dt=1.0, npt=120, pitch=1.0, nx=32, ny=32, dx=1.0, dz=1.0)
    return g.with_blocks(2)


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test collected on a machine without CUDA")
    return torch.device("cuda")
