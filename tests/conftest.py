import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "crowdphot.jl_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 device and the built libcrowdphot_b200.so")


@pytest.fixture(scope="session")
def gpu_ctx():
    import crowdphot_b200 as cpb
    return cpb.get_context(0)
