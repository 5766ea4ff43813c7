import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built engine")
    config.addinivalue_line("markers", "slow: long CPU test")


@pytest.fixture(scope="session")
def ocore():
    import helpers

    return helpers.oracle_core()


@pytest.fixture(scope="session")
def gcore():
    import helpers

    return helpers.pkg.cuda_core()
