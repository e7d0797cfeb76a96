"""GPU parity on the Kelvin-Helmholtz workloads as they are stated, and the
con2prim routines on their own.

The step cases of test_gpu_parity.py run on 64 x 32 grids with a widened
shear layer; here the kernels, called through the C-ABI, are held to the
CPU oracle on the workloads themselves (reference orientation, shear width
a = 0.01):

- the small plain-FP64 workload: 128 x 256 cells, V0 = 0.5, sigma = 1e3,
  MP5 + HLL, SSP2(2,2,2), CFL 0.25, Cardano, 200 steps
  (main_cueva_code.f95:202-289, 16_hll_flow_mpx.f95:735-1979);
- the physics of the 1024 x 2048 benchmark workload in plain FP64: MP5 +
  HLLC, sigma = 1e6, SSP3(4,3,3) with the stage sums reset per stage, on
  128 x 256 cells for 1 and 60 steps and on the full grid for one step
  (11_elecvarint.f95:279-328 at sigma dt = 244);
- whole steps with the Newton-Raphson con2prim (c2p = 0,
  12_varprimitive_nr.f95:6-343);
- cueva_con2prim, the routine mirror of varprimitivecardano and
  varprimitive_nr, point by point against the oracle's routines.

The bars are the reference's: relative L1 per variable <= 1e-12 after one
step and <= 1e-9 after 200 (60 for the four-stage case) in the default
build, which follows the Fortran operation order without FMA contraction.
"""
import os

import numpy as np
import pytest

from conftest import rel_l1_field

pytestmark = pytest.mark.gpu

PRIMS = ["rho", "p", "vx", "vy", "vz", "psi", "phi", "Ex", "Ey", "Ez", "Bx", "By", "Bz", "q"]


def _run_pair(oracle_mod, cfg, checkpoints, c2p=None):
    """Steps the GPU context and the oracle side by side from the workload's
    initial data; asserts the bar at each (steps, bar) checkpoint."""
    from cueva import Cueva
    oracle_mod.set_libm_seed(0)
    oracle_mod.set_threads(os.cpu_count() or 1)
    kw = cfg.solver_kwargs()
    if c2p is not None:
        kw["c2p"] = c2p
    g = Cueva(**kw)
    okw = {k: v for k, v in kw.items() if k != "precision"}
    o = oracle_mod.Oracle(**okw)
    g.kh_init(**cfg.kh_kwargs())
    o.set_prims(g.prims())
    g.upload()
    done = 0
    worst = {}
    for steps, bar in checkpoints:
        g.step(steps - done)
        g.download()
        assert o.step(steps - done) == 0
        done = steps
        ref = o.get_prims()
        for n in PRIMS:
            got = g.interior(n)
            assert np.all(np.isfinite(got)), (steps, n)
            err = rel_l1_field(n, got, ref[n], ref)
            worst[(steps, n)] = err
            assert err <= bar, (steps, n, err)
    g.close()
    return worst


def test_small_workload_as_stated(oracle_mod):
    """128 x 256, MP5 + HLL, SSP2(2,2,2), sigma 1e3, a = 0.01, Cardano:
    1 step <= 1e-12 and 200 steps <= 1e-9 against the oracle."""
    from cueva.configs import C1
    assert (C1.nx, C1.ny, C1.order, C1.flux_solver, C1.rec_mp, C1.c2p, C1.a, C1.sigma) == \
        (128, 256, 2, 5, 0, 1, 0.01, 1e3)
    _run_pair(oracle_mod, C1, [(1, 1e-12), (200, 1e-9)])


def _c2_physics(nx, ny):
    import dataclasses
    from cueva.configs import C2
    return dataclasses.replace(C2, nx=nx, ny=ny, name=C2.name.replace("1024x2048", f"{nx}x{ny}"))


def test_benchmark_physics_fp64_steps(oracle_mod):
    """The benchmark workload's physics (MP5 + HLLC, sigma = 1e6, SSP3(4,3,3)
    with per-stage sum reset, a = 0.01) on 128 x 256 cells: the stiff
    implicit E solve and the HLLC contact in FP64 whole steps, 1 step
    <= 1e-12 and 60 steps <= 1e-9."""
    cfg = _c2_physics(128, 256)
    assert (cfg.order, cfg.flux_solver, cfg.sigma, cfg.intsum_reset, cfg.a) == (4, 7, 1e6, 1, 0.01)
    _run_pair(oracle_mod, cfg, [(1, 1e-12), (60, 1e-9)])


def test_benchmark_workload_full_grid_one_step(oracle_mod):
    """One FP64 step of the 1024 x 2048 benchmark workload itself, <= 1e-12
    per variable against the oracle."""
    _run_pair(oracle_mod, _c2_physics(1024, 2048), [(1, 1e-12)])


@pytest.mark.parametrize("solver,order,rec,reset", [(5, 2, 0, 0), (7, 4, 0, 1), (6, 2, 1, 0), (7, 2, 2, 0)])
def test_newton_raphson_con2prim_steps(oracle_mod, solver, order, rec, reset):
    """c2p = 0 (varprimitive_nr, 12_varprimitive_nr.f95:6-343) in whole
    steps of the 128 x 256 KH layer: 1 step <= 1e-12, 200 steps <= 1e-9.  The
    routine is a one-shot relaxation from the seed p of time n, so the
    result depends on the seed; both sides seed it alike."""
    import dataclasses
    from cueva.configs import C1
    cfg = dataclasses.replace(C1, flux_solver=solver, order=order, rec_mp=rec, intsum_reset=reset, c2p=0)
    _run_pair(oracle_mod, cfg, [(1, 1e-12), (200, 1e-9)], c2p=0)


@pytest.mark.parametrize("method", [1, 0])
def test_con2prim_routine_mirror(oracle_mod, method):
    """cueva_con2prim on the conserved state that varfin leaves after a step
    of the KH layer (D, tau, S), with that step's E and B and the seeds v,
    rho, p of the time level before (main_cueva_code.f95:312-326), equals the
    oracle's varprimitivecardano (method 1) or varprimitive_nr (method 0)
    point by point, bit for bit; the oracle's own step agrees with its
    pointwise routine."""
    from cueva import Cueva
    imax, jmax = 45, 38
    oracle_mod.set_libm_seed(0)
    kw = dict(order=2, flux_solver=5, rec_mp=0, c2p=method, sigma=1e3)
    g = Cueva(imax, jmax, **kw)
    o = oracle_mod.Oracle(imax, jmax, **kw)
    g.kh_init(v0=0.5, a=0.05)
    pr0 = g.prims()
    o.set_prims(pr0)
    assert o.step(3) == 0                     # a state with structure
    pr0 = o.get_prims()
    assert o.step(1) == 0
    pr1 = o.get_prims()
    cons = {n: o.named(n) for n in ("D", "tau", "Sx", "Sy", "Sz")}   # varfin's values
    # the pointwise routine of the oracle: 16 inputs per point
    inp = np.stack([cons["D"], cons["tau"], cons["Sx"], cons["Sy"], cons["Sz"],
                    pr1["Ex"], pr1["Ey"], pr1["Ez"], pr1["Bx"], pr1["By"], pr1["Bz"],
                    pr0["vx"], pr0["vy"], pr0["vz"], pr0["rho"], pr0["p"]], axis=-1)
    want = {n: np.empty(pr1["rho"].shape) for n in ("vx", "vy", "vz", "rho", "p")}
    for j in range(jmax + 1):
        for i in range(imax + 1):
            st, out = oracle_mod.c2p(inp[j, i], method=method, eps1=1e-6)
            assert st == 0, (i, j, st)
            for k, n in enumerate(("vx", "vy", "vz", "rho", "p")):
                want[n][j, i] = out[k]
    for n in want:
        assert np.array_equal(want[n], pr1[n]), n   # the oracle's step uses the same routine
    # the GPU routine mirror on the same inputs
    for n in PRIMS:
        g.set_interior(n, pr1[n] if n not in ("vx", "vy", "vz", "rho", "p") else pr0[n])
    for n, a in (("D", cons["D"]), ("tau", cons["tau"]), ("Sx", cons["Sx"]), ("Sy", cons["Sy"]),
                 ("Sz", cons["Sz"])):
        g.set_interior(n, a)
    g.con2prim()
    for n in want:
        got = g.interior(n)
        nbad = int((got != want[n]).sum())
        assert nbad == 0, f"{n}: {nbad} of {got.size} points differ"
    g.close()


def test_con2prim_biquadratic_state(oracle_mod):
    """cueva_con2prim on the V0 = 0.8 state where the quartic of the Cardano
    recovery is biquadratic to rounding (test_oracle_pins.BIQUAD_STATE): a
    finite result, bit-identical to the oracle's, no status."""
    from test_oracle_pins import BIQUAD_STATE
    from cueva import Cueva
    imax, jmax = 8, 8
    inp = np.array(BIQUAD_STATE)
    g = Cueva(imax, jmax, order=4, flux_solver=7, rec_mp=0, c2p=1, sigma=1e5)
    vals = {"D": inp[0], "tau": inp[1], "Sx": inp[2], "Sy": inp[3], "Sz": inp[4], "Ex": inp[5], "Ey": inp[6],
            "Ez": inp[7], "Bx": inp[8], "By": inp[9], "Bz": inp[10], "vx": inp[11], "vy": inp[12], "vz": inp[13],
            "rho": inp[14], "p": inp[15], "psi": 0.0, "phi": 0.0, "q": 0.0}
    for n, v in vals.items():
        g.set_interior(n, np.full((jmax + 1, imax + 1), v))
    g.con2prim()
    assert g.status() == 0
    st, want = oracle_mod.c2p(inp, method=1, eps1=float(np.float32(1e-6)))
    assert st == 0
    for k, n in enumerate(("vx", "vy", "vz", "rho", "p")):
        got = g.interior(n)
        assert np.all(np.isfinite(got)) and np.all(got == want[k]), n
    g.close()


def test_v08_layer_runs_past_the_biquadratic_state(oracle_mod):
    """The V0 = 0.8, sigma = 1e5 layer (MP5 + HLLC, SSP3(4,3,3) with per-stage
    reset) with a = 0.05 on 256 x 512: the reference's Cardano returned NaN at
    step 5 (point (277, 90)); with the biquadratic limit both sides run on,
    1 step <= 1e-12 and 20 steps <= 1e-9 apart, with no status."""
    import dataclasses
    from cueva.configs import C3
    cfg = dataclasses.replace(C3, nx=256, ny=512, a=0.05, rec_mp=0)
    _run_pair(oracle_mod, cfg, [(1, 1e-12), (20, 1e-9)])
