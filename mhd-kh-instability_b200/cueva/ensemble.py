"""Ensembles of Kelvin-Helmholtz runs advanced by the same launches.

`Ensemble` wraps cueva_ens_*: n independent grids (own size, sigma,
boundaries, time step, con2prim method) that share the scheme (IMEX order,
Riemann solver, reconstruction, precision).  Each RK stage is one y-face
launch and one x-face + update launch over the tiles of every instance, a
step is one CUDA graph, and `autotune()` picks the tile height and the
persistent-grid size by timing them on the ensemble itself.
"""
import ctypes
import math
from dataclasses import dataclass

import numpy as np

from . import _abi

PRIMS = _abi.PRIM_FIELDS


class Ensemble:
    def __init__(self, instances, fma=False):
        """instances: list of keyword dicts as accepted by cueva.Cueva
        (imax, jmax, order, flux_solver, rec_mp, c2p, bc_x, bc_y, precision,
        device, lx, ly, lz, cfl, sigma, gamma, dt, intsum_reset, primitive_rec)."""
        self.L = _abi.load(fma)
        defaults = dict(order=2, flux_solver=5, rec_mp=0, c2p=1, bc_x=0, bc_y=1, precision=0, device=0, lx=2.0,
                        ly=1.0, lz=1.0, cfl=0.25, sigma=1e3, gamma=4.0 / 3.0, dt=0.0, intsum_reset=0,
                        primitive_rec=0)
        self.instances = [dict(defaults, **kw) for kw in instances]
        arr = (_abi.Params * len(self.instances))()
        for k, d in enumerate(self.instances):
            arr[k] = _abi.Params(d["imax"], d["jmax"], d["order"], d["flux_solver"], d["rec_mp"], d["c2p"],
                                 d["bc_x"], d["bc_y"], d["precision"], d["device"], d["intsum_reset"],
                                 d["primitive_rec"], d["lx"],
                                 d["ly"], d["lz"], d["cfl"], d["sigma"], d["gamma"], d["dt"])
        self._params = arr
        h = ctypes.c_void_p()
        _abi.check(self.L, self.L.cueva_ens_create(arr, len(self.instances), ctypes.byref(h)))
        self.h = h

    def __len__(self):
        return len(self.instances)

    def shape(self, k):
        return (self.instances[k]["jmax"] + 1, self.instances[k]["imax"] + 1)

    def kh_init(self, k, v0=0.5, a=0.01, amp=0.01, width=0.01, kpert=2 * math.pi, phase=0.0, bshear=0.1, rho0=1.0,
                p0=1.0):
        _abi.check(self.L, self.L.cueva_ens_kh_init(self.h, k, v0, a, amp, width, kpert, phase, bshear, rho0, p0))

    def get_prims(self, k):
        ny, nx = self.shape(k)
        a = np.empty((len(PRIMS), ny, nx))
        _abi.check(self.L, self.L.cueva_ens_get_prims(self.h, k, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return {n: a[f] for f, n in enumerate(PRIMS)}

    def set_prims(self, k, prims):
        ny, nx = self.shape(k)
        a = np.ascontiguousarray(np.stack([np.asarray(prims[n], dtype=np.float64).reshape(ny, nx) for n in PRIMS]))
        _abi.check(self.L, self.L.cueva_ens_set_prims(self.h, k, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))

    def step(self, n=1):
        _abi.check(self.L, self.L.cueva_ens_step(self.h, int(n)))

    def sync(self):
        """Synchronise; raises CuevaError naming the first failing instance."""
        st = (ctypes.c_uint32 * len(self))()
        rc = self.L.cueva_ens_sync(self.h, st)
        self.status = list(st)
        _abi.check(self.L, rc)
        return self.status

    def set_stream(self, stream_ptr):
        _abi.check(self.L, self.L.cueva_ens_set_stream(self.h, ctypes.c_void_p(stream_ptr)))

    def set_shape(self, rows=8, ctas_per_sm=0):
        _abi.check(self.L, self.L.cueva_ens_set_shape(self.h, rows, ctas_per_sm))

    def autotune(self):
        """Time the launch shapes on the current state, keep the fastest
        (the state is restored); returns (rows, ctas_per_sm, ms per step)."""
        rows, ctas, ms = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_double()
        _abi.check(self.L, self.L.cueva_ens_autotune(self.h, ctypes.byref(rows), ctypes.byref(ctas), ctypes.byref(ms)))
        return rows.value, ctas.value, ms.value

    def attach(self, net):
        _abi.check(self.L, self.L.cueva_ens_attach_mlp(self.h, net.h))

    def set_learned_kernel(self, mode):
        """Learned con2prim: 1 = tcgen05 kernel after the last stage
        (default once attached), 0 = inside the last stage."""
        _abi.check(self.L, self.L.cueva_ens_set_learned_kernel(self.h, int(mode)))

    def learned_stats(self):
        out = (ctypes.c_int64 * 3)()
        _abi.check(self.L, self.L.cueva_ens_learned_stats(self.h, out))
        return list(out)

    def zones(self):
        """Nominal zones (cells) of all instances: sum of imax * jmax."""
        return sum(d["imax"] * d["jmax"] for d in self.instances)

    def close(self):
        if getattr(self, "h", None):
            self.L.cueva_ens_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class KHInstance:
    nx: int        # cells along the flow (periodic) = reference jmax
    ny: int        # cells across the shear layer = reference imax
    v0: float
    a: float
    sigma: float
    bshear: float
    phase: float

    def solver_kwargs(self, **common):
        return dict(common, imax=self.ny, jmax=self.nx, sigma=self.sigma, bc_x=0, bc_y=1, lx=2.0, ly=1.0)

    def kh_kwargs(self):
        return dict(v0=self.v0, a=self.a, amp=0.01, width=0.01, kpert=2 * math.pi, phase=self.phase,
                    bshear=self.bshear, rho0=1.0, p0=1.0)


def kh_ensemble(n=64, seed=2024, nx_choices=(64, 128, 256, 512, 1024)):
    """The batched-ensemble workload: grids nx x 2nx with nx a power of two in
    [64, 1024], V0 uniform [0.1, 0.8], shear width a log-uniform [0.005, 0.05],
    sigma log-uniform [10, 1e6], uniform field uniform [0, 0.3], perturbation
    phase uniform [0, 2 pi), all drawn from numpy's PCG64 with `seed`."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nx = int(rng.choice(nx_choices))
        out.append(KHInstance(nx=nx, ny=2 * nx, v0=float(rng.uniform(0.1, 0.8)),
                              a=float(10 ** rng.uniform(math.log10(0.005), math.log10(0.05))),
                              sigma=float(10 ** rng.uniform(1, 6)), bshear=float(rng.uniform(0.0, 0.3)),
                              phase=float(rng.uniform(0.0, 2 * math.pi))))
    return out
