"""A second, line-by-line restatement of reference routines, pinning the
oracle bit for bit.

The reference cannot be compiled here (no Fortran compiler), so the oracle
(C++) is pinned by properties (test_oracle_pins.py) and, here, against
literal Python transliterations of the Fortran statements of a few routines,
written separately from the oracle: the same arrays, loops and expressions
in the same evaluation order (Python floats are IEEE doubles with correctly
rounded operations, as gfortran's code without -ffast-math).  They cover

- MP5 / MP7 / MP9 (mp5.f95:47-220, mp7.f95, mp9.f95): du and d2, the
  unlimited values vorp / vorm, the median vmpp / vmpm, the limiter with
  DM4 and DMM in the sign arithmetic of funciones.f95:148-185, and the
  positivity fix of the p and rho slots (mp5.f95:177-216);
- get_hllc_vel (funciones.f95:188-259), with the first evaluation at the
  clamped seed (the Fortran reads an uninitialised v there).
"""
import math

import numpy as np
import pytest

G = 6   # ghost cells on each side of a line (-6:n+6)


def f_dsign(a, b):
    """DSIGN(a, b): |a| with the sign of b (the sign bit, so -0d0 gives -|a|)."""
    return math.copysign(abs(a), b)


def f_dmm(x, y):
    """funciones.f95:148-162."""
    return .5 * (f_dsign(1.0, x) + f_dsign(1.0, y)) * min(abs(x), abs(y))


def f_dm4(w, xx, y, z):
    """funciones.f95:165-185."""
    return (.125 * (f_dsign(1.0, w) + f_dsign(1.0, xx))
            * abs((f_dsign(1.0, w) + f_dsign(1.0, y)) * (f_dsign(1.0, w) + f_dsign(1.0, z)))
            * min(abs(w), abs(xx), abs(y), abs(z)))


def _vor(rec, u):
    """vorp / vorm of mp5.f95:62-66, mp7.f95:111-117, mp9.f95:116-123; u(k)
    is the cell at offset k from imp."""
    if rec == 0:
        b1 = 1.0 / 60.0
        vp = b1 * (2.0 * u(-2) - 13.0 * u(-1) + 47.0 * u(0) + 27.0 * u(1) - 3.0 * u(2))
        vm = b1 * (-3.0 * u(-2) + 27.0 * u(-1) + 47.0 * u(0) - 13.0 * u(1) + 2.0 * u(2))
    elif rec == 1:
        b1 = 1.0 / 420.0
        vp = b1 * (-3.0 * u(-3) + 25.0 * u(-2) - 101.0 * u(-1) + 319.0 * u(0) + 214.0 * u(1) - 38.0 * u(2)
                   + 4.0 * u(3))
        vm = b1 * (-3.0 * u(3) + 25.0 * u(2) - 101.0 * u(1) + 319.0 * u(0) + 214.0 * u(-1) - 38.0 * u(-2)
                   + 4.0 * u(-3))
    else:
        b1 = 1.0 / 2520.0
        vp = b1 * (4.0 * u(-4) - 41.0 * u(-3) + 199.0 * u(-2) - 641.0 * u(-1) + 1879.0 * u(0) + 1375.0 * u(1)
                   - 305.0 * u(2) + 55.0 * u(3) - 5.0 * u(4))
        vm = b1 * (4.0 * u(4) - 41.0 * u(3) + 199.0 * u(2) - 641.0 * u(1) + 1879.0 * u(0) + 1375.0 * u(-1)
                   - 305.0 * u(-2) + 55.0 * u(-3) - 5.0 * u(-4))
    return vp, vm


def mp_line_fortran(rec, uline, posfix, stats=None):
    """One line of MP5 / MP7 / MP9 as the Fortran computes it: uline holds
    cells -6 .. n+6; returns up, um on the same cells (set on -2 .. n+2).
    stats, if given, counts the limited values and the positivity fixes."""
    stats = {} if stats is None else stats
    n = uline.size - 2 * G - 1
    mm, nn = 0, n
    alpha_mp, b2, epsm = 2.0, 4.0 / 3.0, 1.0e-10

    def u(i):
        return float(uline[i + G])

    du, d2 = {}, {}
    for imp in range(mm - 5, nn + 6):
        du[imp] = u(imp) - u(imp - 1)
        d2[imp] = u(imp - 1) - 2.0 * u(imp) + u(imp + 1)
    vorp, vorm, vmpp, vmpm = {}, {}, {}, {}
    for imp in range(mm - 2, nn + 3):
        vorp[imp], vorm[imp] = _vor(rec, lambda k: u(imp + k))
        vmpp[imp] = u(imp) + f_dmm(du[imp + 1], alpha_mp * du[imp])
        vmpm[imp] = u(imp) + f_dmm(-du[imp], -alpha_mp * du[imp + 1])
    up = np.zeros_like(uline)
    um = np.zeros_like(uline)
    for imp in range(mm - 2, nn + 3):        # U^L_{i+1/2}, mp5.f95:104-136
        if (vorp[imp] - u(imp)) * (vorp[imp] - vmpp[imp]) <= epsm:
            v = vorp[imp]
        else:
            dm4jph = f_dm4(4.0 * d2[imp] - d2[imp + 1], 4.0 * d2[imp + 1] - d2[imp], d2[imp], d2[imp + 1])
            dm4jmh = f_dm4(4.0 * d2[imp] - d2[imp - 1], 4.0 * d2[imp - 1] - d2[imp], d2[imp], d2[imp - 1])
            vul = u(imp) + alpha_mp * du[imp]
            vav = .5 * (u(imp) + u(imp + 1))
            vmd = vav - .5 * dm4jph
            vlc = u(imp) + .5 * du[imp] + b2 * dm4jmh
            vmin = max(min(u(imp), u(imp + 1), vmd), min(u(imp), vul, vlc))
            vmax = min(max(u(imp), u(imp + 1), vmd), max(u(imp), vul, vlc))
            v = vorp[imp] + f_dmm(vmin - vorp[imp], vmax - vorp[imp])
            stats["limited"] = stats.get("limited", 0) + 1
        up[imp + G] = v
    for imp in range(mm - 2, nn + 3):        # U^R_{i-1/2}, mp5.f95:142-167
        if (vorm[imp] - u(imp)) * (vorm[imp] - vmpm[imp]) <= epsm:
            v = vorm[imp]
        else:
            dm4jph = f_dm4(4.0 * d2[imp] - d2[imp + 1], 4.0 * d2[imp + 1] - d2[imp], d2[imp], d2[imp + 1])
            dm4jmh = f_dm4(4.0 * d2[imp] - d2[imp - 1], 4.0 * d2[imp - 1] - d2[imp], d2[imp], d2[imp - 1])
            vul = u(imp) - alpha_mp * du[imp + 1]
            vav = .5 * (u(imp) + u(imp - 1))
            vmd = vav - .5 * dm4jmh
            vlc = u(imp) - .5 * du[imp + 1] + b2 * dm4jph
            vmin = max(min(u(imp), u(imp - 1), vmd), min(u(imp), vul, vlc))
            vmax = min(max(u(imp), u(imp - 1), vmd), max(u(imp), vul, vlc))
            v = vorm[imp] + f_dmm(vmin - vorm[imp], vmax - vorm[imp])
            stats["limited"] = stats.get("limited", 0) + 1
        um[imp + G] = v
    if posfix:                               # p and rho slots, mp5.f95:177-216
        for imp in range(mm - 2, nn + 3):
            if up[imp + G] < 0.0:
                up[imp + G] = u(imp) + .50 * f_dmm(du[imp], du[imp + 1])
                um[imp + G] = u(imp)
                stats["fixed"] = stats.get("fixed", 0) + 1
        for imp in range(mm - 2, nn + 3):
            if um[imp + G] < 0.0:
                um[imp + G] = u(imp) - .50 * f_dmm(du[imp], du[imp + 1])
                up[imp + G] = u(imp)
                stats["fixed"] = stats.get("fixed", 0) + 1
    return up, um


def _lines(seed, n):
    """Lines that exercise both branches of the limiter and the positivity
    fix: smooth waves, steps, spikes and values near zero."""
    rng = np.random.default_rng(seed)
    x = np.arange(-G, n + G + 1, dtype=np.float64)
    out = [1.0 + 0.3 * np.sin(0.4 * x) + 1e-3 * rng.standard_normal(x.size),
           np.where(x < n / 2, 1.0, 0.125) + 1e-6 * rng.standard_normal(x.size),
           rng.standard_normal(x.size),
           np.abs(rng.standard_normal(x.size)) * (rng.random(x.size) < 0.3) + 1e-12,
           0.02 + 0.05 * np.sign(np.sin(1.3 * x)) * np.abs(np.cos(0.7 * x)),
           np.full(x.size, 0.7)]
    spike = np.full(x.size, 1e-3)
    spike[n // 2 + G] = 5.0
    out.append(spike)
    return out


@pytest.mark.parametrize("rec", [0, 1, 2])
@pytest.mark.parametrize("posfix", [False, True])
def test_mp_line_equals_fortran_statements(oracle_mod, rec, posfix):
    """The oracle's MP line reconstruction equals the literal transliteration
    bit for bit on cells -2 .. n+2 (both limiter branches taken)."""
    n = 40
    k = np.arange(-2, n + 3) + G
    stats = {}
    for seed in range(4):
        for line in _lines(seed, n):
            want_up, want_um = mp_line_fortran(rec, line, posfix, stats)
            got_up, got_um = oracle_mod.mp_line(np.ascontiguousarray(line), rec, posfix)
            assert np.array_equal(got_up[k], want_up[k]), (rec, posfix, seed)
            assert np.array_equal(got_um[k], want_um[k]), (rec, posfix, seed)
    assert stats.get("limited", 0) > 50          # the limiter branch ran
    if posfix:
        assert stats.get("fixed", 0) > 0         # and the positivity fix


def get_hllc_vel_fortran(a, b, c, rt):
    """funciones.f95:188-259; the first pass evaluates f at the clamped seed
    (the Fortran's v is not yet set there).  Returns (v, iterations)."""
    maxiter, minerr, diferr = 100, 1.0e-12, 1.0e-3
    oldv = max(-1.0, min(1.0, rt))
    v = oldv
    it = 0
    while True:
        fv = a * v * v - b * v + c
        dfdv = 2.0 * a * v - b
        v = max(-1.0, min(1.0, oldv - fv / dfdv))
        err = abs(oldv - v)
        oldv = v
        it += 1
        if it >= maxiter:
            return None, it                      # the reference stops here
        if not err > minerr:
            break
    return max(-1.0 + diferr, min(1.0 - diferr, v)), it


def test_hllc_vel_equals_fortran_statements(oracle_mod):
    """The oracle's contact-speed Newton equals the transliteration bit for
    bit on quadratics with a root in (-1, 1), from seeds on both sides."""
    rng = np.random.default_rng(7)
    checked = 0
    for _ in range(3000):
        r = rng.uniform(-0.95, 0.95)
        a = rng.uniform(0.05, 3.0)
        other = r + rng.choice([-1, 1]) * rng.uniform(1.2, 4.0)       # second root outside [-1, 1]
        b = a * (r + other)                                           # a v^2 - b v + c = a (v - r)(v - other)
        c = a * r * other
        rt = rng.uniform(-1.5, 1.5)
        want, it = get_hllc_vel_fortran(a, b, c, rt)
        if want is None:
            continue
        got = oracle_mod.hllc_vel(a, b, c, rt)
        assert got == want, (a, b, c, rt, got, want)
        checked += 1
    assert checked > 2500
