"""Shared test set-up: the ``gpu`` marker, repo root on sys.path, and the library build."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def lib():
    """libcvfes_b200, built in-tree if it is missing (nvcc cross-compiles without a GPU)."""
    from cvfes_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        from cvfes_b200.build import build
        build()
    return _lib.load()


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    return torch.device("cuda", 0)
