import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def built_lib():
    """Path of libhcblas.so, building it in-tree if it is missing."""
    import hcblas_b200
    if not os.path.exists(hcblas_b200.LIB_PATH):
        from hcblas_b200 import build
        build.build()
    return hcblas_b200.LIB_PATH


@pytest.fixture(scope="session")
def handle(built_lib):
    import hcblas_b200 as hb
    s, h = hb.hcblasCreate(0)
    assert s == hb.HCBLAS_STATUS_SUCCESS, f"hcblasCreate failed with status {s}"
    yield h
    hb.hcblasSetMathMode(h, hb.HCBLAS_MATH_NATIVE, 0)
    hb.hcblasDestroy(h)
