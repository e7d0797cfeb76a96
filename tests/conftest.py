import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "mhd-kh-instability_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (ROOT, PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libcueva_b200")


def rel_l1(a, b, floor=1e-15):
    """Relative L1 difference sum|a-b| / sum|b| per variable.

    The denominator is at least floor * size: a variable whose values all sit
    below 1e-15 on an O(0.1-1) state (e.g. the divergence-cleaning potential
    phi of the KH runs, ~1e-38) is round-off noise around an exact zero and is
    compared on that absolute scale instead."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    num = float(np.abs(a - b).sum())
    den = max(float(np.abs(b).sum()), floor * b.size)
    return num / den


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle_py
    oracle_py.build()
    return oracle_py
