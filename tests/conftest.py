import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import __graft_entry__ as ge  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and librn.so")


@pytest.fixture(scope="session")
def rn():
    return ge.load_package()


@pytest.fixture(scope="session")
def oracle():
    return ge.load_oracle()
