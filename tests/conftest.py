import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels")


@pytest.fixture(scope="session")
def oracle():
    from oracle import beta_oracle as bo
    bo.lib()
    return bo


@pytest.fixture(scope="session")
def abi():
    from betanoox_b200 import _abi
    from betanoox_b200.build import build
    build()
    return _abi.load()
