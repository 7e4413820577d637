"""Shared test setup: the `gpu` marker, import paths and common helpers."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libcpsfdtd.so")
    config.addinivalue_line("markers", "slow: longer CPU cases")


def rel_l2(a, b):
    n = np.linalg.norm(b)
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / (n if n > 0 else 1.0))


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    return oracle


@pytest.fixture(scope="session")
def have_ref():
    import oracle
    if not oracle.have_reference_build():
        pytest.skip("reference harness not built (oracle/_ref)")
    return True
