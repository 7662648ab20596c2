import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA builder")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o
    o.build_library()
    return o


@pytest.fixture(scope="session")
def gpu_ctx():
    from marigold_b200 import _lib
    _lib.load()
    return _lib.Context(0)
