"""ctypes wrapper around liboracle.so -- the CPU restatement used as the checker.

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference leg of bench.py.  Nothing in the product imports it.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

PRIM_NAMES = ["rho", "p", "vx", "vy", "vz", "psi", "phi", "Ex", "Ey", "Ez", "Bx", "By", "Bz", "q"]


class OracleParams(ctypes.Structure):
    _fields_ = [("imax", ctypes.c_int32), ("jmax", ctypes.c_int32), ("order", ctypes.c_int32),
                ("flux_solver", ctypes.c_int32), ("rec_mp", ctypes.c_int32), ("c2p", ctypes.c_int32),
                ("bc_x", ctypes.c_int32), ("bc_y", ctypes.c_int32), ("intsum_reset", ctypes.c_int32),
                ("primitive_rec", ctypes.c_int32), ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
                ("cfl", ctypes.c_double), ("sigma", ctypes.c_double), ("gamma", ctypes.c_double),
                ("dt", ctypes.c_double)]


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        L.oracle_create.restype = ctypes.c_void_p
        L.oracle_create.argtypes = [ctypes.POINTER(OracleParams)]
        L.oracle_destroy.argtypes = [ctypes.c_void_p]
        L.oracle_set_threads.argtypes = [ctypes.c_int32]
        L.oracle_set_libm_seed.argtypes = [ctypes.c_int32]
        L.oracle_chebyshev_roots.argtypes = [ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
        L.oracle_cbrt.restype = ctypes.c_double
        L.oracle_cbrt.argtypes = [ctypes.c_double]
        L.oracle_dt.restype = ctypes.c_double
        L.oracle_dt.argtypes = [ctypes.c_void_p]
        L.oracle_set_prims.argtypes = [ctypes.c_void_p, ctypes.POINTER(dp)]
        L.oracle_get_prims.argtypes = [ctypes.c_void_p, ctypes.POINTER(dp)]
        L.oracle_step.restype = ctypes.c_int32
        L.oracle_step.argtypes = [ctypes.c_void_p, ctypes.c_int32]
        L.oracle_run_stages.restype = ctypes.c_int32
        L.oracle_run_stages.argtypes = [ctypes.c_void_p, ctypes.c_int32]
        L.oracle_get_named.restype = ctypes.c_int32
        L.oracle_get_named.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int32, dp]
        L.oracle_get_named_full.restype = ctypes.c_int32
        L.oracle_get_named_full.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int32, dp]
        L.oracle_counters.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)]
        L.oracle_kh_init.argtypes = [ctypes.c_int32, ctypes.c_int32] + [ctypes.c_double] * 11 + \
            [ctypes.POINTER(dp)]
        L.oracle_mp_line.argtypes = [ctypes.c_int32, ctypes.c_int32, dp, ctypes.c_int32, dp, dp]
        L.oracle_hllc_vel.restype = ctypes.c_double
        L.oracle_hllc_vel.argtypes = [ctypes.c_double] * 4
        L.oracle_c2p_cardano.restype = ctypes.c_int32
        L.oracle_c2p_cardano.argtypes = [dp, ctypes.c_double, ctypes.c_double, dp]
        L.oracle_c2p_nr.restype = ctypes.c_int32
        L.oracle_c2p_nr.argtypes = [dp, ctypes.c_double, dp]
        L.oracle_tableau.restype = ctypes.c_int32
        L.oracle_tableau.argtypes = [dp, dp, dp, dp]
        L.oracle_tableau.argtypes = [ctypes.c_int32, dp, dp, dp, dp]
        L.oracle_lector.argtypes = [ctypes.c_void_p] + [ctypes.c_double] * 4 + [ctypes.c_int32, dp, dp]
        _LIB = L
    return _LIB


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ptrs(arrs):
    return (ctypes.POINTER(ctypes.c_double) * len(arrs))(*[_dp(a) for a in arrs])


def set_threads(n):
    lib().oracle_set_threads(int(n))


def set_libm_seed(on):
    """Cardano seed from the C library's acos/cos/pow (1) or the deterministic
    basic-operation seed shared with the kernels (0, default)."""
    lib().oracle_set_libm_seed(int(bool(on)))


class Oracle:
    """One CUEVA run on the host: prims in, prims out, internal arrays by name."""

    def __init__(self, imax, jmax, order=2, flux_solver=5, rec_mp=0, c2p=1, bc_x=0, bc_y=1,
                 lx=2.0, ly=1.0, lz=1.0, cfl=0.25, sigma=1e3, gamma=4.0 / 3.0, dt=0.0, intsum_reset=0,
                 primitive_rec=0):
        self.imax, self.jmax = imax, jmax
        self.p = OracleParams(imax, jmax, order, flux_solver, rec_mp, c2p, bc_x, bc_y, intsum_reset, primitive_rec,
                              lx, ly, lz, cfl, sigma, gamma, dt)
        self.h = lib().oracle_create(ctypes.byref(self.p))
        if not self.h:
            raise ValueError("oracle_create rejected the parameters")

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_destroy(self.h)
            self.h = None

    @property
    def shape(self):
        return (self.jmax + 1, self.imax + 1)   # [j][i], i fastest

    @property
    def dt(self):
        return lib().oracle_dt(self.h)

    def set_prims(self, prims):
        arrs = [np.ascontiguousarray(prims[n], dtype=np.float64).reshape(self.shape) for n in PRIM_NAMES]
        lib().oracle_set_prims(self.h, _ptrs(arrs))

    def get_prims(self):
        arrs = [np.empty(self.shape) for _ in PRIM_NAMES]
        lib().oracle_get_prims(self.h, _ptrs(arrs))
        return dict(zip(PRIM_NAMES, arrs))

    def step(self, n=1):
        return lib().oracle_step(self.h, int(n))

    def run_stages(self, upto):
        return lib().oracle_run_stages(self.h, int(upto))

    def named(self, name, l=1):
        out = np.empty(self.shape)
        if lib().oracle_get_named(self.h, name.encode(), int(l), _dp(out)) != 0:
            raise KeyError(name)
        return out

    def named_full(self, name, l=1):
        """The whole ghosted array, shape (jmax+13, imax+13): element (i, j) at [j+6, i+6]."""
        out = np.empty((self.jmax + 13, self.imax + 13))
        if lib().oracle_get_named_full(self.h, name.encode(), int(l), _dp(out)) != 0:
            raise KeyError(name)
        return out

    def counters(self):
        c = (ctypes.c_int64 * 3)()
        lib().oracle_counters(self.h, c)
        return list(c)

    def lector(self, b0=0.1, lr=3.0, ly=1.0, delta_rec=None, from_startconvar=False):
        """Writer diagnostics (22_writer.f95:821-1019) of the current state:
        (45 values in cueva_diag_slot order, sum |term| of the 35 sums)."""
        if delta_rec is None:
            delta_rec = 1.0e3 ** (-1.0 / 3.0) * lr
        v = np.zeros(45)
        ab = np.zeros(45)
        lib().oracle_lector(self.h, b0, lr, ly, delta_rec, 1 if from_startconvar else 0, _dp(v), _dp(ab))
        return v, ab


def kh_init(imax, jmax, lx=2.0, ly=1.0, v0=0.5, a=0.01, amp=0.01, width=0.01, kpert=2 * np.pi,
            phase=0.0, bshear=0.1, rho0=1.0, p0=1.0):
    arrs = [np.empty((jmax + 1, imax + 1)) for _ in PRIM_NAMES]
    lib().oracle_kh_init(imax, jmax, lx, ly, v0, a, amp, width, kpert, phase, bshear, rho0, p0, _ptrs(arrs))
    return dict(zip(PRIM_NAMES, arrs))


def mp_line(u, rec_mp=0, posfix=False):
    u = np.ascontiguousarray(u, dtype=np.float64)
    n = u.size - 13
    up = np.zeros_like(u)
    um = np.zeros_like(u)
    lib().oracle_mp_line(rec_mp, n, _dp(u), int(posfix), _dp(up), _dp(um))
    return up, um


def hllc_vel(a, b, c, rt):
    return lib().oracle_hllc_vel(a, b, c, rt)


def c2p(inp16, gamma=4.0 / 3.0, method=1, eps1=1e-6):
    inp = np.ascontiguousarray(inp16, dtype=np.float64)
    out = np.zeros(6)
    if method == 1:
        st = lib().oracle_c2p_cardano(_dp(inp), gamma, eps1, _dp(out))
    else:
        st = lib().oracle_c2p_nr(_dp(inp), gamma, _dp(out))
    return st, out


def tableau(order):
    wb, wbt, ab, abt = np.zeros(8), np.zeros(8), np.zeros(64), np.zeros(64)
    s = lib().oracle_tableau(order, _dp(wb), _dp(wbt), _dp(ab), _dp(abt))
    return s, wb, wbt, ab.reshape(8, 8), abt.reshape(8, 8)


def chebyshev_roots(y):
    out = np.zeros(3)
    lib().oracle_chebyshev_roots(float(y), _dp(out))
    return out


def cbrt(x):
    return lib().oracle_cbrt(float(x))
