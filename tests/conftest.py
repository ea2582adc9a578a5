"""Shared fixtures. GPU tests are marked `gpu`; everything else runs on CPU."""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def ref():
    """The reference core compiled from its own sources (oracle/_ref)."""
    from oracle import ref as R
    if not R.available():
        pytest.skip("reference oracle not built and reference sources absent")
    return R


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from neo_fft_b200 import _capi
    _capi.load()
    return torch
