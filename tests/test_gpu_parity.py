"""GPU parity: the sm_100a kernels, called through the C-ABI, against the
CPU oracle on the same inputs.

The default build (libcueva_b200.so, no FMA contraction) follows the Fortran
operation order and the oracle's deterministic Cardano seed, so it must agree
with the oracle to the last bit on finite values; full steps are checked with
the reference's bar, relative L1 per variable <= 1e-12 after one step and
<= 1e-9 after 200 steps.  The FMA build differs in the last bits of every
operation; the reference scheme's limiter switches amplify such differences
in the HLL KH runs (a 1-ulp change of one con2prim seed moves config 1 by
~1e-5 after 200 steps), so for that build the 200-step bar is asserted on the
HLLC case only and the one-step bar on all cases.
"""
import numpy as np
import pytest

from conftest import rel_l1, rel_l1_field

pytestmark = pytest.mark.gpu

PRIMS = ["rho", "p", "vx", "vy", "vz", "psi", "phi", "Ex", "Ey", "Ez", "Bx", "By", "Bz", "q"]
STAGE_MAP = {  # product stage arrays <- oracle arrays of the same stage
    "psiint": "psiint", "phiint": "phiint", "Exint": "Exint", "Eyint": "Eyint", "Ezint": "Ezint",
    "Bxint": "Bxint", "Byint": "Byint", "Bzint": "Bzint", "qint": "qint", "DDint": "DDint",
    "tauint": "tauint", "Sxint": "Sxint", "Syint": "Syint", "Szint": "Szint",
    "Jxint": "Jxint", "Jyint": "Jyint", "Jzint": "Jzint"}
RHS = ["psiflux", "phiflux", "Exastflux", "Eyastflux", "Ezastflux", "Bxflux", "Byflux", "Bzflux", "qflux",
       "Dflux", "tauflux", "Sxflux", "Syflux", "Szflux", "Exastsour", "Eyastsour", "Ezastsour"]


def _pair(oracle_mod, imax, jmax, fma, **kw):
    from cueva import Cueva
    oracle_mod.set_libm_seed(0)
    g = Cueva(imax, jmax, fma=fma, **kw)
    okw = {k: v for k, v in kw.items() if k not in ("precision",)}
    o = oracle_mod.Oracle(imax, jmax, **okw)
    return g, o


def _kh(g, o, v0=0.5, sigma_kw=None):
    g.kh_init(v0=v0)
    pr = g.prims()
    o.set_prims(pr)
    return pr


@pytest.mark.parametrize("solver,rec", [(5, 0), (7, 0), (5, 1), (5, 2), (7, 2), (6, 0), (6, 1), (6, 2), (2, 0), (1, 0), (3, 0), (4, 0)])
def test_flux_rhs_stage1_exact(oracle_mod, solver, rec):
    """hll/hllc_flow_mpx + fluxandsource of stage 1, bit-identical in the default build."""
    imax, jmax = 64, 32
    g, o = _pair(oracle_mod, imax, jmax, False, order=2, flux_solver=solver, rec_mp=rec, sigma=1e3)
    _kh(g, o)
    o.run_stages(1)
    for n, on in STAGE_MAP.items():
        g.set_interior(n, o.named(on), l=1)
    for n in PRIMS:
        g.set_interior(n, o.get_prims()[n])
    g.set_interior("W", o.named("W"))
    g.flux_rhs(1)
    worst = 0.0
    for n in RHS:
        ref = o.named(n, 1)
        got = g.interior(n, 1)
        assert np.all(np.isfinite(got)), n
        diff = np.abs(got - ref)
        scale = max(np.abs(ref).max(), 1e-300)
        worst = max(worst, diff.max() / scale)
        nbad = int((got != ref).sum())
        assert nbad == 0, f"{n}: {nbad} of {got.size} entries differ, max rel {diff.max() / scale:.3e}"
    g.close()


@pytest.mark.parametrize("fma", [False, True])
def test_flux_rhs_stage1_both_builds(oracle_mod, fma):
    imax, jmax = 64, 32
    g, o = _pair(oracle_mod, imax, jmax, fma, order=4, flux_solver=7, rec_mp=0, sigma=1e6)
    _kh(g, o)
    o.run_stages(1)
    for n, on in STAGE_MAP.items():
        g.set_interior(n, o.named(on), l=1)
    for n in PRIMS:
        g.set_interior(n, o.get_prims()[n])
    g.set_interior("W", o.named("W"))
    g.flux_rhs(1)
    for n in RHS:
        assert rel_l1(g.interior(n, 1), o.named(n, 1)) <= 1e-12, n
    g.close()


STEP_CASES = [  # (flux_solver, order, rec_mp, intsum_reset); shear width 0.05 resolves on 64 x 32
    (5, 2, 0, 0), (7, 2, 0, 0), (7, 3, 0, 0), (7, 4, 0, 1), (5, 2, 1, 0), (7, 2, 2, 0), (6, 2, 0, 0), (6, 4, 1, 1),
    (2, 2, 0, 0), (2, 4, 0, 1), (1, 2, 0, 0), (1, 3, 0, 1), (3, 2, 0, 0), (3, 4, 0, 1),
    (4, 2, 0, 0), (4, 4, 0, 1)]


@pytest.mark.parametrize("fma", [False, True])
@pytest.mark.parametrize("solver,order,rec,reset", STEP_CASES)
def test_steps_vs_oracle(oracle_mod, fma, solver, order, rec, reset):
    """Full steps of the fused path: rel L1 <= 1e-12 after 1 step, <= 1e-9 after 200."""
    imax, jmax = 64, 32
    g, o = _pair(oracle_mod, imax, jmax, fma, order=order, flux_solver=solver, rec_mp=rec, sigma=1e3,
                 intsum_reset=reset)
    g.kh_init(v0=0.5, a=0.05)
    o.set_prims(g.prims())
    g.upload()
    g.step(1)
    g.download()
    assert o.step(1) == 0
    ref = o.get_prims()
    for n in PRIMS:
        err = rel_l1_field(n, g.interior(n), ref[n], ref)
        assert err <= 1e-12, (n, err)
    g.step(199)
    g.download()
    assert o.step(199) == 0
    ref = o.get_prims()
    if not fma or (solver, order, rec) == (7, 2, 0):
        for n in PRIMS:
            err = rel_l1_field(n, g.interior(n), ref[n], ref)
            assert err <= 1e-9, (n, err)
    else:
        # chaotic HLL runs: the FMA build rounds differently, and a 1-ulp
        # change of the state grows to ~1e-3 in the velocities and ~1e-2 in
        # the small Bx over 200 steps of this shear layer (how far depends on
        # where the compiler contracts), so only the state's sanity is
        # checked: finite, and within a few per cent of the oracle's
        for n in PRIMS:
            assert np.all(np.isfinite(g.interior(n))) and rel_l1_field(n, g.interior(n), ref[n], ref) <= 5e-2, n
    g.close()


@pytest.mark.parametrize("imax,jmax,solver,rec,bc_x", [
    (45, 38, 7, 0, 0),    # ragged tiles, spacings 2/45 and 1/38 (not powers of two)
    (70, 33, 5, 1, 0),
    (37, 50, 7, 2, 1),    # fully periodic box
    (6, 6, 7, 0, 0),      # smallest grid the ghost maps allow
    (45, 38, 6, 2, 0),    # HLLE
    (45, 38, 2, 0, 0),    # HLL with the MC reconstruction
    (37, 50, 2, 0, 1),
    (45, 38, 1, 0, 0),    # Lax-Friedrichs with MC slopes
    (37, 50, 1, 0, 1),
    (45, 38, 3, 0, 0),    # HLLE with the MC reconstruction
    (37, 50, 3, 0, 1),
    (45, 38, 4, 0, 0),    # HLLC with the MC reconstruction
    (37, 50, 4, 0, 1),
])
def test_steps_ragged_grids(oracle_mod, imax, jmax, solver, rec, bc_x):
    """Partial CTA tiles, non-power-of-two spacings (true divisions in the
    divergence) and both boundary maps: 1 step <= 1e-12, 50 steps <= 1e-9."""
    g, o = _pair(oracle_mod, imax, jmax, False, order=2, flux_solver=solver, rec_mp=rec, sigma=1e3, bc_x=bc_x)
    g.kh_init(v0=0.5, a=0.05)
    o.set_prims(g.prims())
    g.upload()
    for steps, bar in ((1, 1e-12), (49, 1e-9)):
        g.step(steps)
        g.download()
        assert o.step(steps) == 0
        ref = o.get_prims()
        for n in PRIMS:
            err = rel_l1_field(n, g.interior(n), ref[n], ref)
            assert err <= bar, (steps, n, err)
    g.close()


@pytest.mark.parametrize("solver", [5, 7])
def test_ssp433_reference_breakdown_reproduced(oracle_mod, solver):
    """The reference zeroes the stage sums once per step, which makes its
    SSP3(4,3,3) (imex_scheme.f95:278, marked "NO") unstable: the run stops in
    con2prim after a few steps.  The fused path must follow the reference
    step for step: identical prims while the oracle runs, and the con2prim
    status raised at the same step."""
    from cueva import CuevaError
    imax, jmax = 64, 32
    g, o = _pair(oracle_mod, imax, jmax, False, order=4, flux_solver=solver, rec_mp=0, sigma=1e3)
    g.kh_init(v0=0.5, a=0.05)
    o.set_prims(g.prims())
    g.upload()
    for n in range(1, 40):
        st = o.step(1)
        g.step(1)
        if st:
            with pytest.raises(CuevaError):
                g.download()
            assert g.status() & 1
            break
        g.download()
        ref = o.get_prims()
        for f in ("rho", "p", "vx", "vy"):
            assert rel_l1(g.interior(f), ref[f]) <= 1e-10, (n, f)
    else:
        pytest.fail("oracle did not break down")
    g.close()


@pytest.mark.parametrize("solver,order,rec,bc_x,grid", [(7, 2, 0, 0, (64, 32)), (5, 3, 1, 0, (64, 32)),
                                                        (6, 2, 2, 1, (45, 38))])
def test_steps_primitive_reconstruction(oracle_mod, solver, order, rec, bc_x, grid):
    """primitive_rec = 1: every step starts with the diagonal MC
    reconstruction of the primitives (05_reconstruct.f95:525-746) in
    k_recons_begin; 1 step <= 1e-12, 200 steps <= 1e-9 against the oracle."""
    imax, jmax = grid
    g, o = _pair(oracle_mod, imax, jmax, False, order=order, flux_solver=solver, rec_mp=rec, sigma=1e3,
                 bc_x=bc_x, primitive_rec=1)
    g.kh_init(v0=0.5, a=0.05)
    o.set_prims(g.prims())
    g.upload()
    for steps, bar in ((1, 1e-12), (199, 1e-9)):
        g.step(steps)
        g.download()
        assert o.step(steps) == 0
        ref = o.get_prims()
        for n in PRIMS:
            err = rel_l1_field(n, g.interior(n), ref[n], ref)
            assert err <= bar, (steps, n, err)
    g.close()


@pytest.mark.parametrize("solver", [1, 2, 3, 4, 5, 6, 7])
def test_mixed_precision_close_to_fp64_oracle(oracle_mod, solver):
    """precision = 1 (FP32 reconstruction and Riemann solve, FP64 elsewhere)
    for every flux routine: after 1 and 20 steps of the KH layer the
    primitives stay within a small relative L1 of the FP64 oracle -- the
    FP32 rounding of the face fluxes, not a different scheme -- and the run
    raises no status.  Measured on the B200: worst variable after 1 step
    8.3e-7 .. 1.4e-6 for the routines with FP64 field fluxes (all but 3),
    5.6e-6 for HLLE-MC, and 6.1e-6 .. 1.9e-4 after 20
    (Bx, which starts at zero, and the velocities across the shear layer
    grow the rounding fastest)."""
    imax, jmax = 64, 32
    g, o = _pair(oracle_mod, imax, jmax, False, order=2, flux_solver=solver, rec_mp=0, sigma=1e3, precision=1)
    g.kh_init(v0=0.5, a=0.05)
    o.set_prims(g.prims())
    g.upload()
    worst = {}
    for steps, bar in ((1, 2e-5), (19, 1e-3)):
        g.step(steps)
        g.download()
        assert o.step(steps) == 0
        assert g.status() == 0
        ref = o.get_prims()
        for n in PRIMS:
            got = g.interior(n)
            assert np.all(np.isfinite(got)), n
            err = rel_l1_field(n, got, ref[n], ref)
            worst[(steps, n)] = err
            assert err <= bar, (steps, n, err)
    print(f"solver {solver}: worst 1-step {max(v for (s, _), v in worst.items() if s == 1):.2e}, "
          f"20-step {max(v for (s, _), v in worst.items() if s == 19):.2e}")
    g.close()


def _vector_rel_l1(got, ref):
    """Per-variable relative L1, with the components of v, E and B measured
    against the L1 norm of their whole vector (a component that starts at
    zero, such as Bx, has no scale of its own)."""
    out = {n: rel_l1_field(n, got[n], ref[n], ref) for n in PRIMS}
    for comps in (("vx", "vy", "vz"), ("Ex", "Ey", "Ez"), ("Bx", "By", "Bz")):
        den = max(sum(float(np.abs(ref[c]).sum()) for c in comps), 1e-300)
        for c in comps:
            out[c] = float(np.abs(got[c] - ref[c]).sum()) / den
    return out


@pytest.mark.parametrize("solver", [2, 4, 5, 7])   # Lax: vx 1.2e-6 (its FP32 fluid fluxes)
def test_mixed_one_step_within_1e6_on_the_stiff_kh_layer(oracle_mod, solver):
    """Mixed precision on the benchmark's physics (sigma = 1e6, SSP3(4,3,3)
    with per-stage sum reset; MP5 or MC sides): one step stays within relative L1 1e-6 of
    the FP64 oracle for every variable, including Ez and Bx, measured per
    variable and per vector.  The field fluxes carry the uniform B
    background (0.1); in FP32 their rounding alone put Ez at ~3e-6 and Bx
    (per component) at ~5e-5, which the FP64 field fluxes remove."""
    imax, jmax = 256, 128
    g, o = _pair(oracle_mod, imax, jmax, False, order=4, flux_solver=solver, rec_mp=0, sigma=1e6,
                 intsum_reset=1, precision=1)
    g.kh_init(v0=0.5, a=0.01)
    o.set_prims(g.prims())
    g.upload()
    g.step(1)
    g.download()
    assert o.step(1) == 0 and g.status() == 0
    ref = o.get_prims()
    got = {n: g.interior(n) for n in PRIMS}
    per_var = {n: rel_l1_field(n, got[n], ref[n], ref) for n in PRIMS}
    print(f"solver {solver} per variable:", {n: f"{e:.1e}" for n, e in per_var.items() if e > 0})
    for n, e in per_var.items():
        assert e <= 1e-6, (n, e)
    errs = _vector_rel_l1(got, ref)
    print(f"solver {solver}:", {n: f"{e:.1e}" for n, e in errs.items() if e > 0})
    for n, e in errs.items():
        assert e <= 1e-6, (n, e)
    g.close()


# field interface arrays (roles psi, phi, Bn, Bt1, Bt2, En, Et1, Et2), x then y
EB_FACES = ["Exlaxpsi", "Bxlaxphi", "philaxBx", "EzlaxBy", "EylaxBz", "psilaxEx", "BzlaxEy", "BylaxEz",
            "Eylaxpsi", "Bylaxphi", "philaxBy", "ExlaxBz", "EzlaxBx", "psilaxEy", "BxlaxEz", "BzlaxEx"]
# the two of them that carry the uniform By = 0.1 background
BACKGROUND_FACES = ["BylaxEz", "Bylaxphi"]


@pytest.mark.parametrize("solver,rec", [(1, 0), (2, 0), (4, 0), (5, 0), (6, 1), (7, 2)])
def test_mixed_flux_routine_mirror(oracle_mod, solver, rec):
    """cueva_flux_flow of the mixed kernels reads back their scratch layout
    (FP64 slabs for the field roles psi, phi, E, B; FP32 for the rest).
    Errors of the field arrays are measured against the largest field flux
    (some arrays, such as BxlaxEz ~ Ez_R - Ez_L, are differences near zero),
    the fluid arrays against their own size.  The field arrays keep only the
    FP32 rounding of the reconstructed differences (~6e-8 of the local
    variation), so BylaxEz and Bylaxphi, which carry the uniform By = 0.1
    background, agree with the FP64 oracle far below the ~4e-8 that FP32
    rounding of the flux itself gives; the other arrays agree to FP32
    rounding."""
    from cueva import _abi
    imax, jmax = 45, 38
    g, o = _pair(oracle_mod, imax, jmax, False, order=2, flux_solver=solver, rec_mp=rec, sigma=1e3,
                 precision=1)
    _kh(g, o)
    o.run_stages(1)
    for n, on in STAGE_MAP.items():
        g.set_interior(n, o.named(on), l=1)
    for n in PRIMS:
        g.set_interior(n, o.get_prims()[n])
    g.set_interior("W", o.named("W"))
    g.flux_flow(1)
    assert set(EB_FACES) <= set(_abi.FACE_FIELDS)
    refs, gots = {}, {}
    for n in _abi.FACE_FIELDS:
        ref = o.named_full(n)
        refs[n] = ref[6:jmax + 7, 5:imax + 7] if n in _abi.FACE_X else ref[5:jmax + 7, 6:imax + 7]
        gots[n] = g.faces(n, 1)
    fluid = [n for n in _abi.FACE_FIELDS if n.startswith("F")]
    em_scale = max(float(np.abs(refs[n]).max()) for n in _abi.FACE_FIELDS if n not in fluid)
    errs = {}
    for n in _abi.FACE_FIELDS:
        scale = max(float(np.abs(refs[n]).max()), 1e-30) if n in fluid else em_scale
        errs[n] = float(np.abs(gots[n] - refs[n]).max()) / scale
    print(f"solver {solver}: background {max(errs[n] for n in BACKGROUND_FACES):.1e}, "
          f"field worst {max(errs[n] for n in EB_FACES):.1e}, "
          f"others worst {max(e for n, e in errs.items() if n not in EB_FACES):.1e}")
    for n, e in errs.items():
        bar = 5e-9 if n in BACKGROUND_FACES else (1e-8 if n in EB_FACES else 1e-4)
        assert e <= bar, (n, e)
    g.close()


@pytest.mark.parametrize("solver,rec", [(1, 0), (2, 0), (3, 0), (4, 0), (5, 0), (6, 1), (7, 2)])
def test_flux_routine_mirror_interface_fluxes_exact(oracle_mod, solver, rec):
    """cueva_flux_flow is the flux routine alone: its 28 interface flux arrays
    (Exlaxpsi .. FSyzlax) equal the oracle's bit for bit on the faces
    17_fluxandsource.f95 reads, and cueva_fluxandsource on them gives the
    right-hand side of cueva_flux_rhs bit for bit."""
    from cueva import _abi
    imax, jmax = 45, 38   # ragged tiles and non-power-of-two spacings
    g, o = _pair(oracle_mod, imax, jmax, False, order=2, flux_solver=solver, rec_mp=rec, sigma=1e3)
    _kh(g, o)
    o.run_stages(1)
    for n, on in STAGE_MAP.items():
        g.set_interior(n, o.named(on), l=1)
    for n in PRIMS:
        g.set_interior(n, o.get_prims()[n])
    g.set_interior("W", o.named("W"))
    g.flux_flow(1)
    for n in _abi.FACE_FIELDS:
        ref = o.named_full(n)
        ref = ref[6:jmax + 7, 5:imax + 7] if n in _abi.FACE_X else ref[5:jmax + 7, 6:imax + 7]
        got = g.faces(n, 1)
        assert got.shape == ref.shape
        nbad = int((got != ref).sum())
        assert nbad == 0, f"{n}: {nbad} of {got.size} faces differ"
    g.fluxandsource(1)
    split = {n: g.interior(n, 1).copy() for n in RHS}
    g.flux_rhs(1)
    for n in RHS:
        assert np.array_equal(split[n], g.interior(n, 1)), n
        assert np.array_equal(split[n], o.named(n, 1)), n
    g.close()


def test_varfin_electricfield_mirrors(oracle_mod):
    """cueva_varfin / cueva_electricfield: U + Delt * finsum after the last
    stage's sumfin, on the oracle's own final sums and time-n state."""
    imax, jmax = 45, 38
    g, o = _pair(oracle_mod, imax, jmax, False, order=4, flux_solver=7, rec_mp=0, sigma=1e3)
    _kh(g, o)
    o.run_stages(g.lmax)
    fin = {"psi": "psifinsum", "phi": "phifinsum", "Bx": "Bxfinsum", "By": "Byfinsum", "Bz": "Bzfinsum",
           "q": "qfinsum", "D": "Dfinsum", "tau": "taufinsum", "Sx": "Sxfinsum", "Sy": "Syfinsum", "Sz": "Szfinsum",
           "Ex": "Exfinsum", "Ey": "Eyfinsum", "Ez": "Ezfinsum"}
    for n, f in fin.items():
        g.set_interior(f, o.named(f))
        g.set_interior(n, o.named(n))
    g.varfin()
    g.electricfield()
    assert g.dt == o.dt
    for n, f in fin.items():
        assert np.array_equal(g.interior(n), o.named(n) + o.dt * o.named(f)), n
    g.close()


@pytest.mark.parametrize("solver,order,reset,precision", [(7, 4, 1, 0), (5, 2, 0, 0), (6, 2, 0, 0), (2, 4, 1, 0),
                                                          (1, 2, 0, 0), (3, 2, 0, 0), (4, 4, 1, 0), (7, 4, 1, 1),
                                                          (5, 2, 0, 1), (4, 2, 0, 1)])
def test_fused_stage_kernel_equals_split_kernels(solver, order, reset, precision):
    """The fused stage kernel (y faces, x faces and update of a strip in one
    CTA, y fluxes in shared memory) and the two-kernel form (y fluxes through
    device memory) give bit-identical steps, on a grid with ragged strips and
    segments and non-power-of-two spacings, with copy and periodic x."""
    from cueva import Cueva
    for bc_x in (0, 1):
        runs = []
        for fused in (1, 0):
            g = Cueva(93, 70, order=order, flux_solver=solver, rec_mp=0, sigma=1e3, intsum_reset=reset,
                      precision=precision, bc_x=bc_x)
            g.set_stage_kernel(fused)
            assert g.stage_kernel() == fused
            g.kh_init(v0=0.5, a=0.05)
            g.upload()
            g.step(6)
            g.download()
            runs.append({n: g.interior(n).copy() for n in PRIMS})
            g.close()
        for n in PRIMS:
            assert np.array_equal(runs[0][n], runs[1][n]), (bc_x, n)


def test_fused_stage_kernel_refused_without_it():
    from cueva import Cueva, CuevaError
    g = Cueva(64, 32, order=2, flux_solver=7, rec_mp=1)
    assert g.stage_kernel() == 0
    with pytest.raises(CuevaError):
        g.set_stage_kernel(1)
    g.close()
