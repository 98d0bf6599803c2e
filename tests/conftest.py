import importlib
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "golden_cases.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def abi():
    return importlib.import_module("3dnssolver_b200.abi")


@pytest.fixture(scope="session")
def wl():
    return importlib.import_module("3dnssolver_b200.workloads")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


def load_golden():
    z = np.load(GOLDEN)
    meta = json.loads(bytes(z["meta"]).decode())
    return z, meta


def interior(a, g=3):
    return a[g:-g, g:-g, g:-g]


def rel_l2(a, b):
    """Relative L2 error of a against b per conserved field (last axis)."""
    a = a.reshape(-1, a.shape[-1])
    b = b.reshape(-1, b.shape[-1])
    num = np.sqrt(((a - b) ** 2).sum(axis=0))
    den = np.sqrt((b ** 2).sum(axis=0))
    return num / np.maximum(den, 1e-300)
