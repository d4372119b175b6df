import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libcrimson_b200.so")


@pytest.fixture(scope="session")
def small_cyl():
    from crimsonflowsolver_b200 import mesh

    m = mesh.cylinder(ncross=8, naxial=10)
    m.set_inflow(10.0)
    return m


@pytest.fixture(scope="session")
def rng():
    return np.random.default_rng(1234)


def relerr(a, b):
    """max |a-b| / max |b| : the normwise relative error used by the parity tests."""
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))
