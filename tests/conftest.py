import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

GOLDEN = os.path.join(ROOT, "tests", "golden", "golden.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200); runs the CUDA kernels")


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


@pytest.fixture(scope="session")
def sb():
    """The library's Python mirror (stormbitmaps-internal_b200/__init__.py)."""
    return importlib.import_module("stormbitmaps-internal_b200")


def golden_sets(z, prefix):
    import gen
    return gen.from_csr(z[prefix + "vals"], z[prefix + "offs"])
