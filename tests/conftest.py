"""Test configuration: the ``gpu`` marker, and import paths for the package
and the oracle (the oracle is test infrastructure and is used only here,
in ``__graft_entry__.smoke`` and in bench.py's CPU-baseline leg)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path through the C ABI")


def cuda_available() -> bool:
    try:
        import ctypes
        rt = ctypes.CDLL("libcudart.so") if False else None  # noqa: F841
    except OSError:
        pass
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def has_gpu():
    return cuda_available()
