import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "particle-mesh_b200"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def pmpkg():
    from loader import load_package
    return load_package()


@pytest.fixture(scope="session")
def O():
    from oracle import oracle
    return oracle


def golden_cases():
    d = os.path.join(ROOT, "tests", "golden")
    return sorted(f for f in os.listdir(d) if f.endswith(".npz"))


def load_golden(name):
    import numpy as np
    return dict(np.load(os.path.join(ROOT, "tests", "golden", name)))
