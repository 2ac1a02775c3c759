import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


@pytest.fixture(scope="session")
def pkg():
    return importlib.import_module("the-rule-and-compass_b200")


@pytest.fixture(scope="session")
def E(pkg):
    return pkg.expr


@pytest.fixture(scope="session")
def O():
    import oracle
    oracle.lib()
    return oracle
