import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def lai():
    return importlib.import_module("libaccint-public_b200")


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    return o


def golden(name):
    import numpy as np
    return np.load(os.path.join(GOLDEN, name))
