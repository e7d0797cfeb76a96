"""The oracle reproduces its committed fixtures (tests/golden/make_golden.py)
bit for bit: any change of the restated arithmetic shows up here."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def test_oracle_matches_golden(oracle_mod):
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden
    ref = np.load(os.path.join(HERE, "golden", "oracle_kh_small.npz"))
    got = make_golden.compute()
    assert set(ref.files) == set(got)
    for k in ref.files:
        assert np.array_equal(ref[k], got[k], equal_nan=True), k
    # the fixtures are physical (no breakdown) and non-trivial
    for name in make_golden.CASES:
        assert int(ref[f"{name}/status"][0]) == 0
        assert np.abs(ref[f"{name}/rhs1/Sxflux"]).max() > 0
