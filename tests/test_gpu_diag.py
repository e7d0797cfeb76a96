"""GPU: the device-side run diagnostics (the writer's volume integrals and
maxima, 22_writer.f95:821-1019) against the oracle's restatement of the
writer loop, called through the C-ABI.

The terms are computed with the writer's operation order on both sides, so
maxima and point values agree to the bit; the sums are reduced in a
different order (per-thread runs, warp trees, CTA rows) than the writer's
sequential loop, and are held to the summation error bound
|gpu - oracle| <= 2 n u sum|term| (n points, u = 2**-53)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

U = 2.0 ** -53


def _pair(oracle_mod, imax=64, jmax=32, solver=7, order=2, rec=0, **kw):
    from cueva import Cueva
    oracle_mod.set_libm_seed(0)
    g = Cueva(imax, jmax, order=order, flux_solver=solver, rec_mp=rec, sigma=1e3, **kw)
    o = oracle_mod.Oracle(imax, jmax, order=order, flux_solver=solver, rec_mp=rec, sigma=1e3, **kw)
    g.kh_init(v0=0.5, a=0.05)
    o.set_prims(g.prims())
    g.upload()
    return g, o


def _check_record(rec, ref, ab, npts, where):
    from cueva import _abi
    for k, name in enumerate(_abi.DIAG_SLOTS):
        got = rec[name]
        if k < _abi.NDIAG_SUMS:
            bound = 2.0 * npts * U * ab[k] + 1e-300
            assert abs(got - ref[k]) <= bound, (where, name, got, ref[k], bound)
        else:
            assert got == ref[k] or (np.isnan(got) and np.isnan(ref[k])), (where, name, got, ref[k])


@pytest.mark.parametrize("solver,order,rec", [(7, 2, 0), (5, 3, 1), (6, 2, 2)])
def test_records_every_step_match_oracle(oracle_mod, solver, order, rec):
    g, o = _pair(oracle_mod, solver=solver, order=order, rec=rec)
    npts = (g.imax + 1) * (g.jmax + 1)
    g.diag_enable(hglb=1)
    t = 0.0
    for h in range(1, 6):
        g.step(1)
        assert o.step(1) == 0
        t = t + g.dt
        recs = g.diagnostics()
        assert list(recs["h"]) == [h] and recs["t"][0] == t
        ref, ab = o.lector()
        _check_record({k: v[0] for k, v in recs.items()}, ref, ab, npts, h)
    g.close()


def test_record_steps_follow_hglb_and_clock(oracle_mod):
    """h == 1 or mod(h, hglb) == 0, with the clock continued from set_clock."""
    g, o = _pair(oracle_mod)
    g.diag_enable(hglb=3)
    g.step(10)
    assert list(g.diagnostics()["h"]) == [1, 3, 6, 9]
    g.set_clock(20, 1.5)
    g.diag_enable(hglb=5)
    g.step(6)
    r = g.diagnostics()
    assert list(r["h"]) == [25]
    assert r["t"][0] == 1.5 + g.dt + g.dt + g.dt + g.dt + g.dt
    assert g.clock()[0] == 26
    g.close()


def test_capacity_keeps_newest_and_reads_in_chunks(oracle_mod):
    from cueva import _abi
    import ctypes
    g, o = _pair(oracle_mod)
    g.diag_enable(hglb=1, capacity=3)
    g.step(5)
    assert list(g.diagnostics()["h"]) == [3, 4, 5]
    g.step(3)
    buf = (_abi.DiagRecord * 2)()
    n = ctypes.c_int32()
    _abi.check(g.L, g.L.cueva_diag_read(g.ctx, buf, 2, ctypes.byref(n)))
    assert n.value == 2 and [buf[0].h, buf[1].h] == [6, 7]
    assert list(g.diagnostics()["h"]) == [8]
    assert len(g.diagnostics()["h"]) == 0
    g.close()


def test_diag_now_is_startconvar_state(oracle_mod):
    g, o = _pair(oracle_mod, solver=5)
    npts = (g.imax + 1) * (g.jmax + 1)
    g.diag_enable()
    rec = g.diag_now()
    ref, ab = o.lector(from_startconvar=True)
    _check_record(rec, ref, ab, npts, "initial")
    g.step(3)
    assert o.step(3) == 0
    rec = g.diag_now()
    ref, ab = o.lector(from_startconvar=True)
    _check_record(rec, ref, ab, npts, "after 3 steps")
    g.close()


def test_records_leave_the_run_unchanged_and_repeat_bitwise(oracle_mod):
    """A step with a record runs another graph (its last stage also stores
    varfin's D and tau); the state must be bit-identical to a run without
    records, and two runs give bit-identical records."""
    runs = []
    for diag in (False, True, True):
        g, o = _pair(oracle_mod, imax=45, jmax=38)   # ragged tiles
        if diag:
            g.diag_enable(hglb=2)
        g.step(7)
        g.download()
        runs.append((g.prims(), g.diagnostics() if diag else None))
        g.close()
    for n in runs[0][0]:
        assert np.array_equal(runs[0][0][n], runs[1][0][n]), n
    for k, v in runs[1][1].items():
        assert np.array_equal(v, runs[2][1][k]), k


def test_courant_check_does_not_change_dt(oracle_mod):
    g, o = _pair(oracle_mod)
    dt = g.dt
    g.diag_enable(hglb=1)
    g.step(2)
    r = g.diagnostics()
    assert g.dt == dt
    assert np.all(r["max_v"] < 1.0) and np.all(r["max_W"] >= 1.0)
    assert np.all(r["max_lambda_x"] < 1.0) and np.all(r["max_lambda_y"] < 1.0)
    dx, dy = 2.0 / g.imax, 1.0 / g.jmax
    assert np.allclose(r["courant"], dt * np.maximum(r["max_lambda_x"] / dx, r["max_lambda_y"] / dy), rtol=0,
                       atol=0)
    g.close()
