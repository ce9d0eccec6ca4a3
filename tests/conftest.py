import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libhirensi_b200.so")


@pytest.fixture(scope="session")
def gpu_lib():
    """Build (if stale) and load the CUDA library; GPU tests fail loudly without it."""
    from hirensi_b200 import build, capi
    build.build()
    return capi.load()
