"""Learned con2prim seed: training, inference and the comparisons around it.

`LearnedSeed` owns a network of the library (cueva_mlp_*): it is trained on
the GPU by the library's own forward/backward kernels on (conserved,
pressure) pairs -- synthetic states from the seeded generator plus snapshots
of solver runs -- and attached to a `Cueva` context whose params use c2p = 2.
Device buffers are torch tensors (plumbing only; every computation is a
library kernel).  Conserved blocks are (11, n) float64: D, tau, Sx, Sy, Sz,
Ex, Ey, Ez, Bx, By, Bz; primitive blocks (5, n): rho, p, vx, vy, vz.
"""
import ctypes

import numpy as np

from . import _abi

CONS_ORDER = ["D", "tau", "Sx", "Sy", "Sz", "Ex", "Ey", "Ez", "Bx", "By", "Bz"]
PRIM_ORDER = ["rho", "p", "vx", "vy", "vz"]
# batch con2prim methods: Cardano; Newton from the network's seed; Newton from
# given seeds; Newton from the network's seed or the previous pressure,
# whichever leaves the smaller residual (the form the step uses)
CARDANO, NETWORK, SEEDED, BEST = 1, 2, 3, 4


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def synthetic_pairs(n, seed=1234, gamma=4.0 / 3.0, device=0):
    """n synthetic (conserved, primitive) states on the device."""
    import torch
    L = _abi.load()
    cons = torch.empty((11, n), dtype=torch.float64, device=f"cuda:{device}")
    prims = torch.empty((5, n), dtype=torch.float64, device=f"cuda:{device}")
    _abi.check(L, L.cueva_mlp_synthetic_pairs(device, n, seed, gamma, _ptr(cons), _ptr(prims), None))
    torch.cuda.synchronize()
    return cons, prims


def snapshot_pairs(solver):
    """(conserved, primitive) states of a Cueva run's current time level:
    downloads prims and the startconvar group (D, tau, S) of the context."""
    import torch
    solver.download(_abi.G_PRIMS | _abi.G_CONS)
    cons = np.stack([solver.interior(n).ravel() for n in CONS_ORDER])
    prims = np.stack([solver.interior(n).ravel() for n in PRIM_ORDER])
    return torch.from_numpy(cons).cuda(), torch.from_numpy(prims).cuda()


class LearnedSeed:
    def __init__(self, device=0, seed=1234):
        self.L = _abi.load()
        self.device = device
        h = ctypes.c_void_p()
        _abi.check(self.L, self.L.cueva_mlp_create(device, seed, ctypes.byref(h)))
        self.h = h

    # ----------------------------------------------------------- parameters
    def params(self):
        a = np.zeros(_abi.MLP_NPARAM + _abi.MLP_NNORM, dtype=np.float32)
        _abi.check(self.L, self.L.cueva_mlp_get_params(self.h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                       a.size))
        return a

    def set_params(self, a):
        a = np.ascontiguousarray(a, dtype=np.float32)
        _abi.check(self.L, self.L.cueva_mlp_set_params(self.h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                       a.size))

    def save(self, path):
        np.savez(path, params=self.params())

    def load(self, path):
        self.set_params(np.load(path)["params"])

    # -------------------------------------------------------------- training
    def fit_normalisation(self, cons, prims):
        n = cons.shape[1]
        p = prims[1].contiguous()
        _abi.check(self.L, self.L.cueva_mlp_fit_normalisation(self.h, _ptr(cons), _ptr(p), n))

    def train(self, cons, prims, steps=2000, batch=4096, lr=2e-3, seed=99):
        n = cons.shape[1]
        p = prims[1].contiguous()
        loss = ctypes.c_float()
        _abi.check(self.L, self.L.cueva_mlp_train(self.h, _ptr(cons), _ptr(p), n, steps, batch, lr, seed,
                                                  ctypes.byref(loss)))
        return loss.value

    def gradients(self, cons, prims):
        n = cons.shape[1]
        p = prims[1].contiguous()
        g = np.zeros(_abi.MLP_NPARAM, dtype=np.float32)
        loss = ctypes.c_float()
        _abi.check(self.L, self.L.cueva_mlp_gradients(self.h, _ptr(cons), _ptr(p), n,
                                                      g.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                      ctypes.byref(loss)))
        return g, loss.value

    # ------------------------------------------------------------- inference
    def predict(self, cons, tensor_cores=True):
        """Pressure seeds: per-thread FP32 (tensor_cores = False / 0), warp
        mma.sync with bf16 activations (True / 1) or tcgen05 tiles of 128
        states (2, the form the step uses by default)."""
        import torch
        n = cons.shape[1]
        out = torch.empty(n, dtype=torch.float64, device=cons.device)
        mode = int(tensor_cores) if not isinstance(tensor_cores, bool) else (1 if tensor_cores else 0)
        _abi.check(self.L, self.L.cueva_mlp_predict(self.h, _ptr(cons), n, _ptr(out), mode))
        return out

    def c2p(self, method, cons, prev, seed=None, gamma=4.0 / 3.0, eps1=1e-6):
        """Batch con2prim: CARDANO, NETWORK (seed + Newton), SEEDED (Newton
        from `seed`) or BEST (Newton from the network's seed or the previous
        pressure prev[1], whichever has the smaller residual); returns
        (prims (5, n), Newton iterations per state)."""
        import torch
        n = cons.shape[1]
        out = torch.empty((5, n), dtype=torch.float64, device=cons.device)
        it = torch.empty(n, dtype=torch.int32, device=cons.device)
        _abi.check(self.L, self.L.cueva_c2p_batch(self.device, method, self.h, gamma, eps1, _ptr(cons), _ptr(prev),
                                                  _ptr(seed), n, _ptr(out), _ptr(it)))
        return out, it

    def attach(self, solver):
        _abi.check(self.L, self.L.cueva_attach_mlp(solver.ctx, self.h))

    def close(self):
        if getattr(self, "h", None):
            self.L.cueva_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def learned_stats(solver):
    """(Newton iterations, points, Cardano fall-backs) of a context's learned path."""
    out = (ctypes.c_int64 * 3)()
    _abi.check(solver.L, solver.L.cueva_learned_stats(solver.ctx, out))
    return list(out)
