"""Shared pytest configuration: the ``gpu`` marker and common fixtures."""

from __future__ import annotations

from pathlib import Path
import sys

import pytest

REPO = Path(__file__).resolve().parents[1]
GOLDEN = REPO / "tests" / "golden"
for path in (REPO, REPO / "tests"):
    if str(path) not in sys.path:
        sys.path.insert(0, str(path))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a) and the built libolcuda.so")


@pytest.fixture(scope="session")
def native_library():
    """Build (if stale) and load libolcuda.so."""
    from ordinarylight_b200 import _native, build

    from oracle import production

    build.build()
    production.build()
    return _native.load()


@pytest.fixture(scope="session")
def cuda_device():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device; the CUDA renderer has no CPU fallback")
    return torch.device("cuda:0")


@pytest.fixture
def golden():
    import numpy as np

    def load(name):
        return np.load(GOLDEN / name, allow_pickle=False)

    return load
