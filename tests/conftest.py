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

    The denominator is at least floor * size.  Fields that are exactly zero in
    exact arithmetic -- the divergence-cleaning potentials psi, phi and the
    charge q of the 2D KH runs -- only carry round-off (~1e-18..1e-40); for
    them the callers pass the scale of the field they are driven by (the mean
    |E| + |B|), so the comparison is relative to the physics, not to noise."""
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


CLEANING = ("psi", "phi", "q")


def em_scale(prims):
    return float(np.mean(sum(np.abs(prims[n]) for n in ("Ex", "Ey", "Ez", "Bx", "By", "Bz"))))


def rel_l1_field(name, a, b, prims):
    return rel_l1(a, b, em_scale(prims) if name in CLEANING else 1e-15)
