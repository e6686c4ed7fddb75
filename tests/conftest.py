import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU and the built libam24.so")


@pytest.fixture(scope="session")
def am():
    return importlib.import_module("24am_b200")


@pytest.fixture(scope="session")
def po():
    import pyoracle
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        pyoracle.build()
    return pyoracle


@pytest.fixture(scope="session")
def solver(am):
    s = am.Solver(0)
    yield s
    s.close()
