import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def load_golden(key):
    with open(os.path.join(GOLDEN, key + ".json")) as f:
        meta = json.load(f)
    data = dict(np.load(os.path.join(GOLDEN, key + ".npz")))
    return meta, data


def display(field, name):
    """Clamp applied by the reference when it writes a field (PhasePUEq::returnScalar :60-80)."""
    if name == "alpha":
        return np.where(field < 1e-20, 0.0, field)
    if name == "rho":
        return np.where(field < 1e-20, 1e-20, field)
    if name == "tr":  # MeshCartesian::getData src/Meshes/MeshCartesian.cpp:1832-1836
        return np.where(field < 1e-20, 0.0, field)
    return field


def rel_l1(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.abs(b).sum()
    num = np.abs(a - b).sum()
    if den == 0.0:
        return float(num)
    return float(num / den)


@pytest.fixture(scope="session")
def golden_cases():
    from tests.golden.make_golden import golden_cases as g
    return g()
