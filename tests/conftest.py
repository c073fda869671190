"""Shared fixtures.  Tests marked `gpu` need a CUDA device and the built
libillume_gpu.so; everything else runs on the CPU."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built CUDA library")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ctx():
    """One library context on cuda:0 for the GPU tests."""
    import rs_illume_b200 as rb
    c = rb.Context(0)
    yield c
    c.close()
