"""Shared test setup. `-m gpu` tests need a B200 and libmmp_b200.so; everything
else runs on the CPU (oracle checks, host logic, library symbol checks)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU and the built CUDA library")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def mmp():
    """The product library; on a machine with a GPU its absence is an error, not a skip."""
    import mm_propagation_b200 as m
    m.lib()
    return m
