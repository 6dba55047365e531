"""Test configuration: the ``gpu`` marker and in-tree builds of the oracle and native libs."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    from oracle import oracle
    from riv2_b200 import build

    oracle.build()
    build.build_all()
    yield
