"""Asynchronous readback (cueva_download_async) against the synchronous
cueva_download: the same steps through the C-ABI must leave bit-identical host
arrays, whether the next call is an upload of the same arrays (field-ordered
round trip), a step on the device state, or a plain sync.
"""
import numpy as np
import pytest

from cueva import _abi

pytestmark = pytest.mark.gpu

PRIMS = ["rho", "p", "vx", "vy", "vz", "psi", "phi", "Ex", "Ey", "Ez", "Bx", "By", "Bz", "q"]
CONS = ["D", "tau", "Sx", "Sy", "Sz", "W"]


def _make(pinned, imax=96, jmax=64):
    from cueva import Cueva
    g = Cueva(imax, jmax, flux_solver=7, rec_mp=0, sigma=1e3, pinned=pinned)
    g.kh_init(v0=0.5, a=0.05)
    return g


def _snapshot(g, names):
    return {n: g.array(n).copy() for n in names}


@pytest.mark.parametrize("pinned", [True, False])
def test_round_trip_loop_matches_synchronous(pinned):
    """upload -> step -> download_async, repeated: each upload of field f waits
    only for field f's readback, and the result equals the synchronous loop."""
    a, b = _make(pinned), _make(pinned)
    for _ in range(6):
        a.upload()
        a.step(1)
        a.download()
    for _ in range(6):
        b.upload()
        b.step(1)
        b.download_async()
    b.sync()
    for n in PRIMS:
        assert np.array_equal(a.array(n), b.array(n)), n


def test_async_readback_then_steps_and_groups():
    """download_async followed by steps on the device state (the step writes the
    buffers being read back), and of both groups, equals the synchronous path."""
    a, b = _make(True), _make(True)
    a.upload()
    b.upload()
    groups = _abi.G_PRIMS | _abi.G_CONS
    a.step(2)
    a.download(groups)
    ref2 = _snapshot(a, PRIMS + CONS)
    b.step(2)
    b.download_async(groups)
    b.step(3)            # queued after the readback of step 2
    b.sync()
    for n in PRIMS + CONS:
        assert np.array_equal(ref2[n], b.array(n)), n
    a.step(3)
    a.download(groups)
    b.download_async(groups)
    b.download_async(groups)   # a second readback of the same state
    b.sync()
    for n in PRIMS + CONS:
        assert np.array_equal(a.array(n), b.array(n)), n
    assert a.status() == 0 and b.status() == 0


def test_upload_of_conserved_group_after_async_readback():
    """upload(G_PRIMS | G_CONS) right after download_async of both groups: the
    conserved arrays go back up unchanged, and stepping on continues exactly."""
    a, b = _make(True), _make(True)
    groups = _abi.G_PRIMS | _abi.G_CONS
    for g in (a, b):
        g.upload()
        g.step(1)
    a.download(groups)
    a.upload(groups)
    a.step(2)
    a.download()
    b.download_async(groups)
    b.upload(groups)
    b.step(2)
    b.download()
    for n in PRIMS:
        assert np.array_equal(a.array(n), b.array(n)), n


def test_stream_switch_with_pending_readback():
    """set_stream while a readback is in flight: the new stream's work (the
    next step overwrites the buffers being read) waits for the readback."""
    import torch
    a, b = _make(True), _make(True)
    a.upload()
    b.upload()
    a.step(1)
    a.download()
    ref1 = _snapshot(a, PRIMS)
    a.step(1)
    a.download()
    b.step(1)
    b.download_async()
    s = torch.cuda.Stream()
    b.set_stream(s.cuda_stream)
    b.step(1)
    b.sync()
    for n in PRIMS:          # the readback holds step 1, not step 2
        assert np.array_equal(ref1[n], b.array(n)), n
    b.download()
    for n in PRIMS:
        assert np.array_equal(a.array(n), b.array(n)), n
    b.set_stream(None)
