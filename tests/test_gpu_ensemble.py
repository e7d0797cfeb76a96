"""Ensembles: every instance of a batched run must match the same grid run
alone, to the last bit (plain FP64, Cardano), whatever the launch shape."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PRIMS = ["rho", "p", "vx", "vy", "vz", "psi", "phi", "Ex", "Ey", "Ez", "Bx", "By", "Bz", "q"]
GRIDS = [dict(imax=64, jmax=32, sigma=1e3, v0=0.5),
         dict(imax=45, jmax=38, sigma=1e5, v0=0.3),
         dict(imax=128, jmax=64, sigma=30.0, v0=0.6),
         dict(imax=6, jmax=6, sigma=1e3, v0=0.2)]
COMMON = dict(order=4, flux_solver=7, rec_mp=0, intsum_reset=1)


def _single(g, steps):
    from cueva import Cueva
    s = Cueva(g["imax"], g["jmax"], sigma=g["sigma"], **COMMON)
    s.kh_init(v0=g["v0"], a=0.05)
    s.upload()
    s.step(steps)
    s.download()
    out = {n: s.interior(n).copy() for n in PRIMS}
    s.close()
    return out


def _ensemble():
    from cueva.ensemble import Ensemble
    ens = Ensemble([dict(imax=g["imax"], jmax=g["jmax"], sigma=g["sigma"], **COMMON) for g in GRIDS])
    for k, g in enumerate(GRIDS):
        ens.kh_init(k, v0=g["v0"], a=0.05)
    return ens


@pytest.mark.parametrize("rows,ctas", [(8, 0), (4, 0), (8, 1), (4, 3)])
def test_ensemble_matches_single_runs(rows, ctas):
    steps = 5
    ens = _ensemble()
    ens.set_shape(rows, ctas)
    ens.step(steps)
    ens.sync()
    for k, g in enumerate(GRIDS):
        ref = _single(g, steps)
        got = ens.get_prims(k)
        for n in PRIMS:
            assert np.array_equal(got[n], ref[n]), (k, n, float(np.abs(got[n] - ref[n]).max()))
    ens.close()


def test_autotune_keeps_the_state():
    ens = _ensemble()
    rows, ctas, ms = ens.autotune()
    assert rows in (4, 8) and ctas >= 0 and ms > 0
    ens.step(5)
    ens.sync()
    for k, g in enumerate(GRIDS):
        ref = _single(g, 5)
        got = ens.get_prims(k)
        for n in PRIMS:
            assert np.array_equal(got[n], ref[n]), (k, n)
    ens.close()


def test_ensemble_rejects_mixed_schemes():
    """Instances share the scheme: differing stage-sum conventions are refused."""
    from cueva import CuevaError
    from cueva.ensemble import Ensemble
    inst = [dict(imax=64, jmax=32, sigma=1e3, order=4, flux_solver=7, intsum_reset=r) for r in (1, 0)]
    with pytest.raises(CuevaError):
        Ensemble(inst)


def test_learned_ensemble_matches_single_runs():
    """Instances with the learned con2prim (c2p = 2, network attached) next
    to Cardano ones: the tcgen05 con2prim launch covers the learned
    instances' tiles only, and every instance matches its single run to the
    bit (same tiles of 128 points, same MMAs)."""
    from cueva import Cueva
    from cueva.ensemble import Ensemble
    from cueva.learned import LearnedSeed, synthetic_pairs
    cons, prims = synthetic_pairs(100_000, seed=99)
    net = LearnedSeed(seed=5)
    net.fit_normalisation(cons, prims)
    net.train(cons, prims, steps=300, batch=4096, lr=2e-3)
    c2ps = [2, 1, 2, 2]
    ens = Ensemble([dict(imax=g["imax"], jmax=g["jmax"], sigma=g["sigma"], c2p=c, **COMMON)
                    for g, c in zip(GRIDS, c2ps)])
    for k, g in enumerate(GRIDS):
        ens.kh_init(k, v0=g["v0"], a=0.05)
    ens.attach(net)
    ens.step(4)
    ens.sync()
    for k, (g, c) in enumerate(zip(GRIDS, c2ps)):
        s = Cueva(g["imax"], g["jmax"], sigma=g["sigma"], c2p=c, **COMMON)
        s.kh_init(v0=g["v0"], a=0.05)
        s.upload()
        net.attach(s)
        s.step(4)
        s.download()
        got = ens.get_prims(k)
        for n in PRIMS:
            assert np.array_equal(got[n], s.interior(n)), (k, n)
        s.close()
    ens.close()
    net.close()


def test_primitive_reconstruction_ensemble_matches_single_runs():
    from cueva import Cueva
    from cueva.ensemble import Ensemble
    common = dict(COMMON, primitive_rec=1)
    ens = Ensemble([dict(imax=g["imax"], jmax=g["jmax"], sigma=g["sigma"], **common) for g in GRIDS])
    for k, g in enumerate(GRIDS):
        ens.kh_init(k, v0=g["v0"], a=0.05)
    ens.step(4)
    ens.sync()
    for k, g in enumerate(GRIDS):
        s = Cueva(g["imax"], g["jmax"], sigma=g["sigma"], **common)
        s.kh_init(v0=g["v0"], a=0.05)
        s.upload()
        s.step(4)
        s.download()
        got = ens.get_prims(k)
        for n in PRIMS:
            assert np.array_equal(got[n], s.interior(n)), (k, n)
        s.close()
    ens.close()


@pytest.mark.parametrize("solver,precision", [(1, 0), (1, 1), (2, 0), (3, 1), (4, 0), (4, 1), (6, 1), (7, 1)])
def test_ensemble_other_flux_routines_match_single_runs(solver, precision):
    """The batched path runs every flux routine (and the mixed-precision
    kernels, whose FP64 field-flux slabs sit at offsets of each instance's
    own scratch stride) exactly like single runs."""
    from cueva import Cueva
    from cueva.ensemble import Ensemble
    common = dict(COMMON, flux_solver=solver, precision=precision)
    ens = Ensemble([dict(imax=g["imax"], jmax=g["jmax"], sigma=g["sigma"], **common) for g in GRIDS])
    for k, g in enumerate(GRIDS):
        ens.kh_init(k, v0=g["v0"], a=0.05)
    ens.step(3)
    ens.sync()
    for k, g in enumerate(GRIDS):
        s = Cueva(g["imax"], g["jmax"], sigma=g["sigma"], **common)
        s.kh_init(v0=g["v0"], a=0.05)
        s.upload()
        s.step(3)
        s.download()
        got = ens.get_prims(k)
        for n in PRIMS:
            assert np.array_equal(got[n], s.interior(n)), (solver, k, n)
        s.close()
    ens.close()
