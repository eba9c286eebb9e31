import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def mf():
    return importlib.import_module("mille-feillue_b200")


@pytest.fixture(scope="session")
def O():
    import _oracle

    return _oracle


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tiles_ref.npz")
    z = np.load(path)
    cases = {}
    for key in z.files:
        case, name = key.split("/", 1)
        cases.setdefault(case, {})[name] = z[key]
    return cases
