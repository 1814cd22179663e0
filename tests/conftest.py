import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a); runs the kernels through the C-ABI")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.build(ref=False)
    return oracle


@pytest.fixture(scope="session")
def lib():
    import libspimage_b200 as L

    if not os.path.exists(L.LIB_PATH):
        from libspimage_b200 import build

        build.build()
    L.load()
    assert L.load().spb_device_count() > 0, "no CUDA device visible"
    return L
