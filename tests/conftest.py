import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_sessionstart(session):
    """Build the CUDA library in-tree if it is missing (nvcc cross-compiles
    without a GPU); a GPU machine uses the prebuilt file."""
    lib = os.path.join(ROOT, "lela_b200", "liblela_cuda.so")
    if not os.path.exists(lib):
        from lela_b200 import build
        build.build()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (runs the CUDA path)")
    config.addinivalue_line("markers", "slow: long-running test")


@pytest.fixture(scope="session")
def cuda():
    """One CUDA-module handle for the whole GPU session (fails loudly when
    the library or the device is missing)."""
    import lela_b200
    m = lela_b200.CudaModule(0)
    yield m
    m.close()
