import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libmcmax_gpu.so")


@pytest.fixture(scope="session")
def ctx():
    from mcmax_b200 import api
    c = api.Context(0)
    yield c
    c.close()
