"""Regenerates tests/golden/oracle_kh_small.npz: outputs of the CPU oracle on
small KH cases (prims after a few steps for several solver / reconstruction /
con2prim / boundary / primitive-reconstruction combinations, all seven flux
routines, and the stage-1 right-hand side).

The reference ships no golden vectors and cannot be compiled here, so these
fixtures pin the oracle against its own regressions; test_golden.py checks the
current oracle reproduces them bit for bit.  Run from the repository root:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

CASES = {
    # name: (imax, jmax, oracle kwargs, kh kwargs, steps)
    "hll_ssp222_mp5": (32, 16, dict(order=2, flux_solver=5, rec_mp=0, c2p=1), dict(v0=0.5, a=0.1), 4),
    "hllc_ssp332_mp7": (32, 16, dict(order=3, flux_solver=7, rec_mp=1, c2p=1, sigma=1e5), dict(v0=0.6, a=0.1), 3),
    "hll_ssp222_mp9_nr": (32, 16, dict(order=2, flux_solver=5, rec_mp=2, c2p=0), dict(v0=0.4, a=0.1), 3),
    "hllc_ssp433_reset_periodic": (24, 24, dict(order=4, flux_solver=7, rec_mp=0, c2p=1, bc_x=1, bc_y=1,
                                                lx=1.0, ly=1.0, intsum_reset=1, sigma=1e6),
                                   dict(v0=0.3, a=0.1, lx=1.0, ly=1.0), 3),
    "hlle_ssp222_mp7": (32, 16, dict(order=2, flux_solver=6, rec_mp=1, c2p=1), dict(v0=0.5, a=0.1), 3),
    "lax_ssp222": (32, 16, dict(order=2, flux_solver=1, c2p=1), dict(v0=0.5, a=0.1), 4),
    "hll_mc_ssp332": (32, 16, dict(order=3, flux_solver=2, c2p=1), dict(v0=0.5, a=0.1), 3),
    "hlle_mc_ssp222_nr": (32, 16, dict(order=2, flux_solver=3, c2p=0), dict(v0=0.5, a=0.1), 3),
    "hllc_mc_ssp433_periodic": (24, 24, dict(order=4, flux_solver=4, c2p=1, bc_x=1, bc_y=1, lx=1.0, ly=1.0,
                                             sigma=1e5), dict(v0=0.3, a=0.1, lx=1.0, ly=1.0), 3),
    "hllc_primrec_ssp222": (32, 16, dict(order=2, flux_solver=7, rec_mp=0, c2p=1, primitive_rec=1),
                            dict(v0=0.5, a=0.1), 3),
}
RHS = ["psiflux", "phiflux", "Exastflux", "Eyastflux", "Ezastflux", "Bxflux", "Byflux", "Bzflux", "qflux",
       "Dflux", "tauflux", "Sxflux", "Syflux", "Szflux", "Exastsour", "Eyastsour", "Ezastsour"]


def compute():
    import oracle_py
    oracle_py.build()
    oracle_py.set_threads(4)
    out = {}
    for name, (imax, jmax, okw, khkw, steps) in CASES.items():
        pr = oracle_py.kh_init(imax, jmax, **khkw)
        o = oracle_py.Oracle(imax, jmax, **okw)
        o.set_prims(pr)
        o.run_stages(1)
        for n in RHS:
            out[f"{name}/rhs1/{n}"] = o.named(n, 1)
        o2 = oracle_py.Oracle(imax, jmax, **okw)
        o2.set_prims(pr)
        st = o2.step(steps)
        out[f"{name}/status"] = np.array([st])
        for n, a in o2.get_prims().items():
            out[f"{name}/prims/{n}"] = a
    return out


if __name__ == "__main__":
    data = compute()
    np.savez_compressed(os.path.join(HERE, "oracle_kh_small.npz"), **data)
    print(f"wrote {len(data)} arrays")
