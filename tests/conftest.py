import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); calls through the C ABI of libefl_b200.so")


@pytest.fixture(scope="session")
def oracle_api():
    from oracle import py_oracle
    return py_oracle.load()


@pytest.fixture(scope="session")
def gpu_api():
    from bevy_eulerian_fluid_b200 import _capi
    return _capi.load()
