"""Shared pytest set-up: the `gpu` marker, imports of the package (directory name has a dash) and of the oracle."""
import importlib
import os
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.dirname(__file__))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def hb():
    return importlib.import_module("honee-4aiad_b200")


@pytest.fixture(scope="session")
def prob():
    return importlib.import_module("honee-4aiad_b200.problem")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.build()
    return O
