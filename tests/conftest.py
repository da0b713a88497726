import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA library")


def _load(name):
    with np.load(os.path.join(GOLDEN, name)) as d:
        return {k: d[k] for k in d.files}


@pytest.fixture(scope="session")
def gsc():
    return _load("golden_sc.npz")


@pytest.fixture(scope="session")
def gsq():
    return _load("golden_sq.npz")


@pytest.fixture(scope="session")
def ggrad():
    return _load("golden_grad.npz")


def relmax(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="session")
def gamg():
    return _load("golden_amg.npz")
