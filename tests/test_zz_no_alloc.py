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


@pytest.mark.parametrize("solver,rec,precision", [(7, 0, 0), (5, 2, 0), (7, 0, 1), (5, 2, 1)])
def test_noalloc_matches_flux_rhs(oracle_mod, solver, rec, precision):
    """precision = 1 runs the mixed kernels, whose scratch holds FP64 slabs
    for the field roles and FP32 slabs for the rest; the reference call is
    cueva_flux_rhs of a context with the same precision."""
    torch = pytest.importorskip("torch")
    from cueva import Cueva, _abi
    imax, jmax = 64, 32
    oracle_mod.set_libm_seed(0)
    g = Cueva(imax, jmax, order=2, flux_solver=solver, rec_mp=rec, sigma=1e3, precision=precision)
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


def test_noalloc_refuses_a_capturing_stream():
    """The call uploads its descriptor from its own stack and may wait for
    the stream, so a stream under capture is refused before anything is
    enqueued."""
    torch = pytest.importorskip("torch")
    from cueva import _abi
    L = _abi.load()
    imax, jmax = 64, 32
    p = _abi.Params(imax, jmax, 2, 7, 0, 1, 0, 1, 0, 0, 0, 0, 2.0, 1.0, 1.0, 0.25, 1e3, 4.0 / 3.0, 0.0)
    pitch, ny = 72, jmax + 1
    prim = torch.zeros((14, ny, pitch), dtype=torch.float64, device="cuda")
    W = torch.ones((1, ny, pitch), dtype=torch.float64, device="cuda")
    stage = torch.zeros((17, ny, pitch), dtype=torch.float64, device="cuda")
    rhs = torch.zeros((17, ny, pitch), dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.stream(s):
        graph.capture_begin()
        rc = L.cueva_flux_rhs_noalloc(ctypes.byref(p), prim.data_ptr(), W.data_ptr(), stage.data_ptr(),
                                      rhs.data_ptr(), pitch, pitch * ny, s.cuda_stream, None)
        rhs.add_(0.0)   # keeps the captured graph non-empty
        graph.capture_end()
    assert rc == _abi.CUEVA_ERR_ARG
    assert b"captured" in L.cueva_last_error()
    del graph
