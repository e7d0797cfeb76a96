"""Pins of the CPU oracle (the checker): analytic and structural properties of
the restated Fortran that must hold whatever the reference would print.

The reference ships no tests or golden vectors and cannot be compiled here
(no Fortran compiler), so these are the anchors of the restatement."""
import numpy as np
import pytest

from conftest import rel_l1


def _line(vals):
    return np.ascontiguousarray(vals, dtype=np.float64)


@pytest.mark.parametrize("rec", [0, 1, 2])
def test_mp_linear_exact(oracle_mod, rec):
    n = 24
    x = np.arange(-6, n + 7, dtype=np.float64)
    u = 0.3 + 0.7 * x
    up, um = oracle_mod.mp_line(_line(u), rec)
    k = np.arange(-2, n + 3) + 6
    np.testing.assert_allclose(up[k], 0.3 + 0.7 * (x[k] + 0.5), rtol=0, atol=1e-13)
    np.testing.assert_allclose(um[k], 0.3 + 0.7 * (x[k] - 0.5), rtol=0, atol=1e-13)


@pytest.mark.parametrize("rec,deg", [(0, 4), (1, 6), (2, 8)])
def test_mp_polynomial_exact(oracle_mod, rec, deg):
    """Unlimited MP5/7/9 interface values are exact for cell averages of
    polynomials of degree <= 4/6/8; a gentle monotone polynomial keeps the
    limiter off (SH97 eq. 2.1/2.31)."""
    n, h = 32, 1.0 / 64
    rng = np.random.default_rng(7 + rec)
    coef = rng.uniform(-0.3, 0.3, deg + 1) * (0.2 ** np.arange(deg + 1))
    coef[1] = 1.0
    P = np.polynomial.Polynomial(coef)
    Pi = P.integ()
    xe = (np.arange(-6, n + 8) - 0.5) * h          # cell edges
    avg = (Pi(xe[1:]) - Pi(xe[:-1])) / h            # cell averages of cells -6..n+6
    up, um = oracle_mod.mp_line(_line(avg), rec)
    k = np.arange(-2, n + 3) + 6
    xc = (np.arange(-6, n + 7)) * h
    np.testing.assert_allclose(up[k], P(xc[k] + 0.5 * h), rtol=0, atol=2e-12)
    np.testing.assert_allclose(um[k], P(xc[k] - 0.5 * h), rtol=0, atol=2e-12)


@pytest.mark.parametrize("rec", [0, 1, 2])
@pytest.mark.parametrize("posfix", [False, True])
def test_mp_odd_symmetry_bitwise(oracle_mod, rec, posfix):
    """MP5/7/9 are odd: the reference's separately reconstructed -E/-B slots
    equal the negated E/B values bit for bit (basis of the kernels' shortcut).
    The p/rho positivity fix is not odd, so only posfix=False is compared."""
    rng = np.random.default_rng(11 + rec)
    u = rng.standard_normal(40 + 13).cumsum() * 0.1 + rng.standard_normal(53) * 0.5
    up, um = oracle_mod.mp_line(_line(u), rec, posfix)
    upn, umn = oracle_mod.mp_line(_line(-u), rec, posfix)
    k = np.arange(-2, 40 + 3) + 6
    if not posfix:
        assert np.array_equal(upn[k], -up[k]) and np.array_equal(umn[k], -um[k])
    else:
        assert np.all(np.isfinite(up[k]))


def test_mp_positivity_fix(oracle_mod):
    """p/rho slots never reconstruct negative values next to positive cells
    (mp5.f95:177-216)."""
    u = np.full(40 + 13, 1.0)
    u[20:] = 1e-6        # strong jump that overshoots below zero unlimited
    up, um = oracle_mod.mp_line(_line(u), 0, True)
    k = np.arange(-2, 43) + 6
    assert (up[k] >= 0).all() and (um[k] >= 0).all()


def test_hllc_vel_root(oracle_mod):
    rng = np.random.default_rng(3)
    for _ in range(200):
        v = rng.uniform(-0.9, 0.9)
        a = rng.uniform(0.5, 2.0)
        w = rng.uniform(1.5, 4.0) * np.sign(rng.standard_normal())  # second root outside [-1, 1]
        # a (x - v)(x - w) = a x^2 - a (v + w) x + a v w = a x^2 - b x + c
        b, c = a * (v + w), a * v * w
        got = oracle_mod.hllc_vel(a, b, c, v + 0.05)
        assert abs(got - v) < 1e-10


def _random_prims(rng, n):
    rho = 10 ** rng.uniform(-1, 1, n)
    p = 10 ** rng.uniform(-2, 1, n)
    W = rng.uniform(1.0, 3.0, n)
    vdir = rng.standard_normal((n, 3))
    vdir /= np.linalg.norm(vdir, axis=1)[:, None]
    v = vdir * np.sqrt(1 - 1 / W ** 2)[:, None]
    B = rng.standard_normal((n, 3)) * 0.5
    E = -np.cross(v, B) + rng.standard_normal((n, 3)) * 1e-3
    return rho, p, v, E, B


def _cons(rho, p, v, E, B, gamma=4 / 3):
    V2 = (v ** 2).sum(1)
    W = 1 / np.sqrt(1 - V2)
    h = rho * (1 + p / ((gamma - 1) * rho)) + p
    D = rho * W
    tau = 0.5 * ((E ** 2).sum(1) + (B ** 2).sum(1)) + h * W ** 2 - p
    S = np.cross(E, B) + (h * W ** 2)[:, None] * v
    return D, tau, S


@pytest.mark.parametrize("method", [1, 0])
def test_c2p_round_trip(oracle_mod, method):
    """prim -> cons -> prim: Cardano recovers the primitives to ~1e-9 from a
    seed at the true state (the reference seeds with the time-n prims)."""
    rng = np.random.default_rng(5)
    rho, p, v, E, B = _random_prims(rng, 300)
    D, tau, S = _cons(rho, p, v, E, B)
    worst = 0.0
    for k in range(300):
        inp = np.r_[D[k], tau[k], S[k], E[k], B[k], v[k], rho[k], p[k]]
        st, out = oracle_mod.c2p(inp, method=method)
        assert st == 0
        if method == 1:
            worst = max(worst, abs(out[3] / rho[k] - 1), abs(out[4] / p[k] - 1),
                        np.abs(out[:3] - v[k]).max())
    assert worst < 1e-8


def test_tableaux_consistent(oracle_mod):
    for order in (1, 2, 3, 4, 5, 6, 8):
        s, wb, wbt, ab, abt = oracle_mod.tableau(order)
        assert s >= 1
        # IMEX-RK48SSP stores rational approximations that sum to 1 - 1.2e-7
        assert abs(wb.sum() - 1) < 1e-6 and abs(wbt[:s].sum() - (0 if order == 1 else 1)) < 1e-6
        if order != 1:   # order 1 stores Ab(1,1) = 1, never read (sumint runs m = 1..l-1)
            assert np.all(np.triu(ab[:s, :s]) == 0)             # explicit part strictly lower
        assert np.all(np.triu(abt[:s, :s], 1) == 0)             # implicit part lower (DIRK)


@pytest.mark.parametrize("solver,order,rec", [(5, 2, 0), (7, 4, 0), (7, 2, 1), (5, 3, 2), (6, 2, 0), (6, 4, 2), (2, 2, 0),
                                              (2, 4, 0), (1, 2, 0), (1, 4, 0), (3, 2, 0),
                                              (3, 4, 0), (4, 2, 0), (4, 4, 0)])
def test_uniform_state_stays_uniform(oracle_mod, solver, order, rec):
    imax, jmax = 20, 12
    o = oracle_mod.Oracle(imax, jmax, order=order, flux_solver=solver, rec_mp=rec, bc_x=0, bc_y=1, sigma=1e3)
    v = np.array([0.3, -0.2, 0.1])
    B = np.array([0.1, 0.2, -0.05])
    E = -np.cross(v, B)
    shape = (jmax + 1, imax + 1)
    pr = {"rho": np.full(shape, 1.3), "p": np.full(shape, 0.7), "psi": np.zeros(shape), "phi": np.zeros(shape),
          "q": np.zeros(shape)}
    for c, n in enumerate("xyz"):
        pr["v" + n] = np.full(shape, v[c])
        pr["E" + n] = np.full(shape, E[c])
        pr["B" + n] = np.full(shape, B[c])
    o.set_prims(pr)
    assert o.step(3) == 0
    out = o.get_prims()
    for n, a in out.items():
        # round-off of the stiff source sigma W (E + v x B ...) is amplified by sigma
        np.testing.assert_allclose(a, pr[n], rtol=1e-11, atol=1e-13, err_msg=n)


def test_periodic_mass_conservation(oracle_mod):
    """Fully periodic box: the flux divergence telescopes, so sum(D) over the
    unique points changes only by the con2prim tolerance."""
    imax, jmax = 24, 24
    o = oracle_mod.Oracle(imax, jmax, order=2, flux_solver=5, bc_x=1, bc_y=1, lx=1.0, ly=1.0, sigma=1e3)
    pr = oracle_mod.kh_init(imax, jmax, lx=1.0, ly=1.0, v0=0.3, a=0.1)
    o.set_prims(pr)
    o.run_stages(0)
    d0 = o.named("D")[:-1, :-1].sum()
    o2 = oracle_mod.Oracle(imax, jmax, order=2, flux_solver=5, bc_x=1, bc_y=1, lx=1.0, ly=1.0, sigma=1e3)
    o2.set_prims(pr)
    o2.step(5)
    o2.run_stages(0)
    d1 = o2.named("D")[:-1, :-1].sum()
    assert abs(d1 / d0 - 1) < 1e-9


def test_implicit_e_residual(oracle_mod):
    """electricvarint solves E - E* + a W (E + v x B - (E.v) v) = 0 with a = Abt(l,l) sigma dt."""
    imax, jmax = 32, 16
    sigma = 1e6
    o = oracle_mod.Oracle(imax, jmax, order=2, flux_solver=5, sigma=sigma)
    pr = oracle_mod.kh_init(imax, jmax)
    pr["Ex"] = pr["Ex"] + 1e-3 * np.sin(np.arange(pr["Ex"].size)).reshape(pr["Ex"].shape)
    o.set_prims(pr)
    o.run_stages(1)
    s, wb, wbt, ab, abt = oracle_mod.tableau(2)
    a = abt[0, 0] * sigma * o.dt
    W = o.named("W")
    E = np.stack([o.named("Exint"), o.named("Eyint"), o.named("Ezint")], -1)
    Ea = np.stack([o.named("Exast"), o.named("Eyast"), o.named("Ezast")], -1)
    B = np.stack([o.named("Bxint"), o.named("Byint"), o.named("Bzint")], -1)
    v = np.stack([pr["vx"], pr["vy"], pr["vz"]], -1)
    Edv = (E * v).sum(-1)
    res = E - Ea + (a * W)[..., None] * (E + np.cross(v, B) - Edv[..., None] * v)
    scale = np.abs(Ea).max() + np.abs(E).max()
    assert np.abs(res).max() < 1e-12 * max(1.0, a) * max(scale, 1e-3)


def test_threads_bit_identical(oracle_mod):
    imax, jmax = 40, 20
    outs = []
    for nt in (1, 4):
        oracle_mod.set_threads(nt)
        o = oracle_mod.Oracle(imax, jmax, order=4, flux_solver=7, sigma=1e4)
        o.set_prims(oracle_mod.kh_init(imax, jmax))
        o.step(3)
        outs.append(o.get_prims())
    oracle_mod.set_threads(8)
    for n in outs[0]:
        assert np.array_equal(outs[0][n], outs[1][n]), n


def test_kh_init_matches_formula(oracle_mod):
    imax, jmax = 16, 8
    pr = oracle_mod.kh_init(imax, jmax, v0=0.5, a=0.01)
    x = -1.0 + np.arange(imax + 1) * (2.0 / imax)
    y = -0.5 + np.arange(jmax + 1) * (1.0 / jmax)
    X, Y = np.meshgrid(x, y)
    np.testing.assert_allclose(pr["vy"], 0.5 * np.tanh(X / 0.01), rtol=1e-15, atol=1e-16)
    np.testing.assert_allclose(pr["vx"], 0.01 * np.sin(2 * np.pi * Y) * np.exp(-(X * X) / 0.01), atol=1e-17)
    np.testing.assert_allclose(pr["Ez"], -(pr["vx"] * 0.1), rtol=1e-15)
    assert rel_l1(pr["By"], np.full_like(pr["By"], 0.1)) == 0


def test_cardano_seed_helpers_match_libm(oracle_mod):
    """The deterministic seed arithmetic equals the C library's
    cos((acos y + 2 pi k)/3) and x**(1/3) to a few ulp."""
    rng = np.random.default_rng(9)
    for y in np.r_[rng.uniform(-0.999999, 0.999999, 500), -0.5, 0.0, 0.5]:
        t = np.arccos(y)
        ref = np.cos(np.array([t, t + 2 * np.pi, t - 2 * np.pi]) / 3)
        got = oracle_mod.chebyshev_roots(y)
        # both sides are ill-conditioned next to the double roots y = +-1
        assert np.abs(got - ref).max() < 4e-15 / (1 - abs(y)) ** 0.5, y
    # x**THIRD of the reference is the cube root to within |ln x| * 1.9e-17
    for x in np.r_[10 ** rng.uniform(-300, 300, 500), 1.0, 8.0, 27.0]:
        assert abs(oracle_mod.cbrt(x) / np.cbrt(x) - 1) < 4e-16
    assert oracle_mod.cbrt(0.0) == 0.0


@pytest.mark.parametrize("solver", [5, 7])
def test_seed_modes_agree_after_one_step(oracle_mod, solver):
    """C-library and deterministic Cardano seeds give the same step to the
    last few bits (they differ by ~1 ulp in W only)."""
    imax, jmax = 64, 32
    outs = []
    for libm in (1, 0):
        oracle_mod.set_libm_seed(libm)
        o = oracle_mod.Oracle(imax, jmax, order=2, flux_solver=solver, sigma=1e3)
        o.set_prims(oracle_mod.kh_init(imax, jmax, a=0.05))
        assert o.step(1) == 0
        outs.append(o.get_prims())
    oracle_mod.set_libm_seed(0)
    for n in outs[0]:
        assert rel_l1(outs[0][n], outs[1][n]) <= 1e-14, n


def test_c2p_status_codes(oracle_mod):
    """Fault injection on the CPU: conserved states that the reference's
    con2prim stops on raise the documented status bits instead (Cardano
    `stop` sites = bit 1); the NR form returns non-finite values, which the
    step's wrapper reports as bit 16."""
    inp = np.zeros(16)
    inp[[0, 1, 2, 14, 15]] = [1.0, 1.0, 5.0, 1.0, 1.0]          # |S| > tau: no physical state
    st, out = oracle_mod.c2p(inp, method=1)
    assert st & 1
    st, out = oracle_mod.c2p(inp, method=0)
    assert not np.all(np.isfinite(out))
    inp[[1, 2]] = [-1.0, 0.0]                                     # negative energy
    st, out = oracle_mod.c2p(inp, method=1)
    assert st & 1
    good = np.array([1.2, 2.0, 0.1, 0, 0, 0, 0, 0, 0, 0.1, 0, 0, 0, 0, 1, 1], dtype=float)
    st, out = oracle_mod.c2p(good, method=1)
    assert st == 0 and np.all(np.isfinite(out))


def test_primitive_reconstruction_is_identity_to_rounding(oracle_mod):
    """05_reconstruct.f95 (primitive_rec = 1) takes the same limiter
    arguments for the R and L values of a point, so (R + L)/2 returns the
    value up to the rounding of (u - x) + (u + x): a uniform state stays
    exact, a KH state changes by a few ulp."""
    pr = oracle_mod.kh_init(32, 16, v0=0.5, a=0.05)
    runs = {}
    for r in (0, 1):
        o = oracle_mod.Oracle(32, 16, order=2, flux_solver=7, primitive_rec=r)
        o.set_prims(pr)
        assert o.step(1) == 0
        runs[r] = o.get_prims()
    for n in runs[0]:
        a, b = runs[0][n], runs[1][n]
        scale = max(float(np.abs(a).max()), 1e-300)
        assert float(np.abs(a - b).max()) <= 1e-14 * scale, n
    u = {n: np.full_like(v, 0.25 if n in ("rho", "p") else 0.0) for n, v in pr.items()}
    o = oracle_mod.Oracle(32, 16, order=2, flux_solver=5, primitive_rec=1)
    o.set_prims(u)
    assert o.step(1) == 0
    out = o.get_prims()
    for n in u:
        assert np.array_equal(out[n], u[n]), n


def test_mcl_reconstruction_second_order(oracle_mod):
    """The MC reconstruction of flux_solver 2 (16_hll_flow_mcl.f95) is exact
    on linear data away from extrema, and its "_m" values negate only the
    cell value: -u + slope, not -(u + slope)."""
    pr = oracle_mod.kh_init(24, 12, v0=0.0, a=0.05, amp=0.0)
    ramp = np.add.outer(0.01 * np.arange(13), 0.02 * np.arange(25)) + 1.0   # linear in i and j
    pr = {n: (ramp.copy() if n in ("rho", "p") else np.zeros_like(ramp)) for n in pr}
    o = oracle_mod.Oracle(24, 12, order=1, flux_solver=2, bc_x=0, bc_y=0, sigma=1.0)
    o.set_prims(pr)
    assert o.run_stages(1) == 0
    # the x flux of D at interior faces is 0.5 (FD_L + FD_R) - 0.5 (D_R - D_L) with v = 0:
    # -(D_R - D_L)/2 with the exact face values, i.e. 0 for continuous linear data
    fd = o.named("FDxlax", 1)
    assert np.allclose(fd[2:-2, 2:-3], 0.0, atol=1e-14)


def test_lax_right_state_takes_the_slopes_of_p(oracle_mod):
    """flux_solver 1 (15_lax_flow.f95:920-1457): each cell carries
    p = F + U and m = F - U, and the right state of a face is
    m(i+1) - FAC mcl(p(i+2) - p(i+1), p(i+1) - p(i)) -- the slopes of p,
    not of m.  With v = 0 the D flux F = D vx vanishes, so on data linear in
    the cell index (step a) the face flux is 0.5 (D + a/2 - D - 3a/2) = -a/2,
    where slopes of m would give 0."""
    imax, jmax = 24, 12
    pr = oracle_mod.kh_init(imax, jmax, v0=0.0, a=0.05, amp=0.0)
    ramp = np.add.outer(0.01 * np.arange(jmax + 1), 0.02 * np.arange(imax + 1)) + 1.0
    pr = {n: (ramp.copy() if n in ("rho", "p") else np.zeros_like(ramp)) for n in pr}
    o = oracle_mod.Oracle(imax, jmax, order=1, flux_solver=1, bc_x=0, bc_y=0, sigma=1.0)
    o.set_prims(pr)
    assert o.run_stages(1) == 0
    fdx, fdy = o.named("FDxlax", 1), o.named("FDylax", 1)
    assert np.allclose(fdx[:, 1:-2], -0.01, rtol=0, atol=1e-14)
    assert np.allclose(fdy[1:-2, :], -0.005, rtol=0, atol=1e-14)
    # the charge flux pairs J with q: both vanish here
    assert np.all(o.named("Jxlax", 1) == 0.0)


def _uniform_prims(imax, jmax):
    v = np.array([0.3, -0.2, 0.1])
    B = np.array([0.1, 0.2, -0.05])
    E = -np.cross(v, B)
    shape = (jmax + 1, imax + 1)
    pr = {"rho": np.full(shape, 1.3), "p": np.full(shape, 0.7), "psi": np.zeros(shape), "phi": np.zeros(shape),
          "q": np.zeros(shape)}
    for c, n in enumerate("xyz"):
        pr["v" + n] = np.full(shape, v[c])
        pr["E" + n] = np.full(shape, E[c])
        pr["B" + n] = np.full(shape, B[c])
    return pr, v, E, B


@pytest.mark.parametrize("solver", [1, 2, 3, 4, 5, 6, 7])
def test_interface_flux_consistent_on_uniform_state(oracle_mod, solver):
    """F(U, U) = F(U): on a uniform state every flux routine returns the
    physical flux of the state on every face (the Maxwell, cleaning and
    fluid parts; the sign-flipped arrays EzlaxBy / BylaxEz / ExlaxBz /
    BzlaxEx hold -F) -- except the reference's own HLLE-MC energy flux, which
    is pinned to its closed form instead."""
    imax, jmax = 16, 12
    pr, v, E, B = _uniform_prims(imax, jmax)
    o = oracle_mod.Oracle(imax, jmax, order=1, flux_solver=solver, bc_x=0, bc_y=1, sigma=1e3)
    o.set_prims(pr)
    assert o.run_stages(1) == 0
    gam = 4.0 / 3.0
    rho, p = 1.3, 0.7
    W = 1.0 / np.sqrt(1.0 - v @ v)
    h = rho * (1.0 + p / ((gam - 1.0) * rho)) + p
    # stage-1 E is the implicit solve of E = -v x B, which returns it up to rounding
    Ex, Ey, Ez = (o.named(n)[0, 0] for n in ("Exint", "Eyint", "Ezint"))
    D = rho * W
    expect = {
        "Exlaxpsi": Ex, "Eylaxpsi": Ey, "Bxlaxphi": B[0], "Bylaxphi": B[1], "philaxBx": 0.0, "philaxBy": 0.0,
        "psilaxEx": 0.0, "psilaxEy": 0.0, "EylaxBz": Ey, "EzlaxBx": Ez, "EzlaxBy": Ez, "ExlaxBz": Ex,
        "BzlaxEy": B[2], "BxlaxEz": B[0], "BylaxEz": B[1], "BzlaxEx": B[2],
        "FDxlax": D * v[0], "FDylax": D * v[1],
        "Ftauxlax": (B[2] * Ey - B[1] * Ez) + h * W**2 * v[0],
        "Ftauylax": (B[0] * Ez - B[2] * Ex) + h * W**2 * v[1],
        "FSxylax": -Ex * Ey - B[0] * B[1] + h * W**2 * v[0] * v[1],
    }
    if solver == 3:
        # the reference's HLLE-MC star energy (16_hlle_flow_mcl.f95, taustr_*)
        # is not consistent: on a uniform state with v* = vn,
        # tau*_L = tau - |E,B|^2/2 vn/(vn - s1) and tau*_R = tau + |E,B|^2/2 vn/(s2 - vn),
        # so the star flux F + s (tau* - tau) is off by that much (s1, s2 the
        # HLLE bounds, with the reference's vn under the root)
        Cs = np.sqrt(gam * p / h)
        V2 = v @ v
        eb2 = 0.5 * ((Ex**2 + Ey**2 + Ez**2) + (B @ B))
        for name, vn in (("Ftauxlax", v[0]), ("Ftauylax", v[1])):
            root = np.sqrt((1.0 - V2) * (1.0 - V2 * Cs**2 - vn * (1.0 - Cs**2)))
            s1 = (vn * (1.0 - Cs**2) - Cs * root) / (1.0 - Cs**2 * V2)
            s2 = (vn * (1.0 - Cs**2) + Cs * root) / (1.0 - Cs**2 * V2)
            assert s1 < 0.0 < s2
            expect[name] += (-s1 * eb2 * vn / (vn - s1)) if vn >= 0.0 else (s2 * eb2 * vn / (s2 - vn))
    for name, val in expect.items():
        got = o.named(name)[1:-1, 1:-1]
        np.testing.assert_allclose(got, val, rtol=1e-12, atol=1e-14, err_msg=f"{solver} {name}")


def test_hllc_em_fluxes_equal_hll(oracle_mod):
    """HLLC (flux_solver 7) keeps the HLL fluxes of the Maxwell equations
    (16_hllc_flow_mpx.f95 star EM fluxes are the HLL ones), bit for bit; only
    psi, phi and the fluid fluxes receive the contact correction."""
    imax, jmax = 32, 16
    pr = oracle_mod.kh_init(imax, jmax, v0=0.5, a=0.05)
    arrs = {}
    for solver in (5, 7):
        o = oracle_mod.Oracle(imax, jmax, order=1, flux_solver=solver, sigma=1e3)
        o.set_prims(pr)
        assert o.run_stages(1) == 0
        arrs[solver] = {n: o.named(n) for n in ("philaxBx", "EzlaxBy", "EylaxBz", "psilaxEx", "BzlaxEy", "BylaxEz",
                                                 "EzlaxBx", "philaxBy", "ExlaxBz", "BzlaxEx", "psilaxEy", "BxlaxEz",
                                                 "FDxlax")}
    for n in arrs[5]:
        if n == "FDxlax":
            assert not np.array_equal(arrs[5][n], arrs[7][n]), n   # corrected by the contact
        else:
            assert np.array_equal(arrs[5][n], arrs[7][n]), n


# A state of the V0 = 0.8 KH layer (256 x 512, a = 0.05, step 5, point
# (277, 90)) where the depressed quartic of the Cardano recovery is
# biquadratic to rounding (d_1 = 3e-9): d_2 + 2 z_1 of the one-real-root
# branch comes out as -1.3e-15.  Exact bits; D, tau, S, E, B, then the seeds.
BIQUAD_STATE = [float.fromhex(h) for h in (
    "0x1.7dcd0bb9e7a81p+0", "0x1.442aaecbba2e9p+3", "-0x1.7bf2784f7b54cp-5", "0x1.0830b1d8ae4d0p+3", "0x0.0p+0",
    "0x0.0p+0", "0x0.0p+0", "0x1.ba9505f926cc5p-12", "0x1.300b04ea65465p-17", "0x1.9976c538ce886p-4", "0x0.0p+0",
    "-0x1.101b440068168p-8", "0x1.7bf60cdc988bep-1", "0x0.0p+0", "0x1.ffd74b35d9abcp-1", "0x1.ffc9c1aa05e5bp-1")]


def test_cardano_biquadratic_state_recovered(oracle_mod):
    """Where the reference's square root of d_2 + 2 z_1 would take a
    rounding-level negative argument (a silent NaN in 12_varprimitive.f95),
    the recovery takes the biquadratic limit: a finite state whose conserved
    variables reproduce the input, and that agrees with the NR recovery."""
    inp = np.array(BIQUAD_STATE)
    st, out = oracle_mod.c2p(inp, method=1, eps1=float(np.float32(1e-6)))
    assert st == 0 and np.all(np.isfinite(out))
    vx, vy, vz, rho, p, W = out
    D, tau, S = _cons(np.array([rho]), np.array([p]), np.array([[vx, vy, vz]]), inp[None, 5:8], inp[None, 8:11])
    assert abs(D[0] / inp[0] - 1) < 1e-9 and abs(tau[0] / inp[1] - 1) < 1e-9
    assert np.abs(S[0] - inp[2:5]).max() < 1e-9 * np.abs(inp[2:5]).max()
    st_nr, out_nr = oracle_mod.c2p(inp, method=0)
    assert st_nr == 0 and abs(out_nr[3] / rho - 1) < 1e-4 and abs(out_nr[1] / vy - 1) < 1e-4
