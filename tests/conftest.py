import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def params():
    from comer2_b200 import params as P
    return P.load_default()


@pytest.fixture(scope="session")
def orc32(params):
    from oracle_py import Oracle
    return Oracle(params, 32)


@pytest.fixture(scope="session")
def orc64(params):
    from oracle_py import Oracle
    return Oracle(params, 64)
