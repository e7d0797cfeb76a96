"""Error measures used to compare two runs of the same workload.

rel_l1(a, b) = sum|a - b| / sum|b| per variable.  The divergence-cleaning
potentials psi, phi and the charge q of the 2D Kelvin-Helmholtz runs are zero
in exact arithmetic and only carry round-off; for them the denominator is the
scale of the fields that drive them (mean |E| + |B| per point), so the number
is relative to the physics rather than to noise.
"""
import numpy as np

CLEANING = ("psi", "phi", "q")


def rel_l1(a, b, floor=1e-15):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    num = float(np.abs(a - b).sum())
    den = max(float(np.abs(b).sum()), floor * b.size)
    return num / den


def em_scale(prims):
    return float(np.mean(sum(np.abs(prims[n]) for n in ("Ex", "Ey", "Ez", "Bx", "By", "Bz"))))


def rel_l1_field(name, a, b, prims):
    """rel_l1 of variable `name`; prims holds the reference run's fields."""
    return rel_l1(a, b, em_scale(prims) if name in CLEANING else 1e-15)
