"""cueva_flux_rhs_noalloc against cueva_flux_rhs.

The no-allocation entry point takes device arrays from the caller and keeps
its interface-flux scratch in a fixed block of static device memory.  Its
stage right-hand side must match the context-based routine mirror on the same
inputs, on two calls in a row (the second call reuses the scratch the first
one left behind).  The file name sorts last so that the test also runs after
every other GPU test in one session; it passes alone in a fresh process too.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PRIMS = ["rho", "p", "vx", "vy", "vz", "psi", "phi", "Ex", "Ey", "Ez", "Bx", "By", "Bz", "q"]
STAGE = ["psiint", "phiint", "Exint", "Eyint", "Ezint", "Bxint", "Byint", "Bzint", "qint", "DDint", "tauint",
         "Sxint", "Syint", "Szint", "Jxint", "Jyint", "Jzint"]
RHS = ["psiflux", "phiflux", "Exastflux", "Eyastflux", "Ezastflux", "Bxflux", "Byflux", "Bzflux", "qflux",
       "Dflux", "tauflux", "Sxflux", "Syflux", "Szflux", "Exastsour", "Eyastsour", "Ezastsour"]


def _device_group(torch, arrays, pitch, ny):
    """Pack interior arrays (ny, nx) into one device slab of len(arrays) fields."""
    nx = arrays[0].shape[1]
    slab = torch.zeros((len(arrays), ny, pitch), dtype=torch.float64, device="cuda")
    for f, a in enumerate(arrays):
        slab[f, :, :nx] = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return slab


@pytest.mark.parametrize("solver,rec", [(7, 0), (5, 2)])
def test_noalloc_matches_flux_rhs(oracle_mod, solver, rec):
    torch = pytest.importorskip("torch")
    from cueva import Cueva, _abi
    imax, jmax = 64, 32
    oracle_mod.set_libm_seed(0)
    g = Cueva(imax, jmax, order=2, flux_solver=solver, rec_mp=rec, sigma=1e3)
    o = oracle_mod.Oracle(imax, jmax, order=2, flux_solver=solver, rec_mp=rec, sigma=1e3)
    g.kh_init(v0=0.5, a=0.05)
    o.set_prims(g.prims())
    o.run_stages(1)
    for n in STAGE:
        g.set_interior(n, o.named(n), l=1)
    for n in PRIMS:
        g.set_interior(n, o.get_prims()[n])
    g.set_interior("W", o.named("W"))
    g.flux_rhs(1)                                    # the existing entry point
    want = {n: g.interior(n, 1).copy() for n in RHS}

    nx, ny = imax + 1, jmax + 1
    pitch = 72                                       # any pitch >= imax + 1
    prim = _device_group(torch, [g.interior(n) for n in PRIMS], pitch, ny)
    W = _device_group(torch, [g.interior("W")], pitch, ny)
    stage = _device_group(torch, [g.interior(n, 1) for n in STAGE], pitch, ny)
    fstride = pitch * ny
    L = g.L
    for call in range(2):
        rhs = torch.full((len(RHS), ny, pitch), float("nan"), dtype=torch.float64, device="cuda")
        st = ctypes.c_uint32(0)
        torch.cuda.synchronize()
        rc = L.cueva_flux_rhs_noalloc(ctypes.byref(g.params), prim.data_ptr(), W.data_ptr(), stage.data_ptr(),
                                      rhs.data_ptr(), pitch, fstride, torch.cuda.current_stream().cuda_stream,
                                      ctypes.byref(st))
        _abi.check(L, rc)
        assert st.value == 0
        got = rhs[:, :, :nx].cpu().numpy()
        for f, n in enumerate(RHS):
            ref = want[n]
            err = np.abs(got[f] - ref).sum() / max(np.abs(ref).sum(), 1e-300)
            assert np.all(np.isfinite(got[f])), (call, n)
            assert err <= 1e-12, (call, n, err)
    g.close()


def test_noalloc_rejects_oversized_grid():
    from cueva import _abi
    L = _abi.load()
    p = _abi.Params(4096, 4096, 2, 7, 0, 1, 0, 1, 0, 0, 0, 0, 2.0, 1.0, 1.0, 0.25, 1e3, 4.0 / 3.0, 0.0)
    st = ctypes.c_uint32(0)
    dummy = ctypes.c_void_p(16)
    rc = L.cueva_flux_rhs_noalloc(ctypes.byref(p), dummy, dummy, dummy, dummy, 4097, 4097 * 4097, None,
                                  ctypes.byref(st))
    assert rc == _abi.CUEVA_ERR_ARG
    assert b"too large" in L.cueva_last_error()
