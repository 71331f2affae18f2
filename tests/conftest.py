"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device and the built libmmb200.so; all
others run on CPU (oracle, golden fixtures, host logic, library exports)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built CUDA library")


@pytest.fixture(scope="session")
def golden():
    """The reference's golden fields (tests/golden/ref_fields.npz, from src/magnum_tests/ref)."""
    d = np.load(os.path.join(ROOT, "tests", "golden", "ref_fields.npz"))
    return {k: d[k] for k in d.files}


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.restated()
    return oracle


@pytest.fixture(scope="session")
def ref_available(oracle_mod):
    return oracle_mod.have_reference()


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def unit_random(rng, n):
    v = rng.normal(size=(3, n))
    return v / np.linalg.norm(v, axis=0)
