import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    O.lib()
    return O


@pytest.fixture(scope="session")
def cuda_lib():
    """The sm_100a library, loaded (built first if absent). GPU tests use it."""
    from splat_b200 import _native as N
    from splat_b200 import build

    if not os.path.exists(N.LIB_PATH):
        build.build()
    return N.lib()
