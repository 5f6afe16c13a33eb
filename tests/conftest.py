import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    from oracle import pyoracle
    pyoracle.build()
    from godar_b200 import build
    build.build_gen()
    if not os.path.exists(build.LIB):
        build.build_gpu()
    yield
