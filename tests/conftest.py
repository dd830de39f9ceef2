import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the product's kernels")


@pytest.fixture(scope="session")
def fdtd():
    """The product binding; building it first if needed (nvcc cross-compiles without a GPU)."""
    import fdtd3d_b200
    from fdtd3d_b200 import build

    build.build()
    fdtd3d_b200.load_library()
    return fdtd3d_b200
