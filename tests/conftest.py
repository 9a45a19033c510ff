import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the library's kernels")


@pytest.fixture(scope="session")
def ctx():
    """One device context for the GPU tests (device 0)."""
    import wadjet_b200 as wg
    c = wg.Context(0)
    yield c
    c.close()
