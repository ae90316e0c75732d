import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: large inputs (seconds of CPU oracle time)")


@pytest.fixture(scope="session")
def ctx():
    from fastmulticolsort_b200 import capi
    c = capi.Context(0)
    yield c
    c.close()
