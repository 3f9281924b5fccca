import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built librcb200.so")


def _have_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def built_lib():
    """Path of the in-tree shared library, building it when missing (CPU-side nvcc)."""
    from rayleighchebyshevgpgpu_b200 import build
    if not os.path.exists(build.LIB_PATH):
        build.build()
    return build.LIB_PATH


@pytest.fixture(scope="session")
def ctx(built_lib):
    if not _have_gpu():
        pytest.fail("GPU test selected but no CUDA device is visible")
    from rayleighchebyshevgpgpu_b200.runtime import Context
    c = Context(0)
    yield c
    c.close()
