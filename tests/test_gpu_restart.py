"""GPU: restarts.  A run continued from a binary checkpoint, or from the
reference's text backup (all_variables_NNNN.dat) written and read by the
library, is bit-identical to the uninterrupted run; bad checkpoints are
refused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ctx(**kw):
    from cueva import Cueva
    base = dict(order=2, flux_solver=7, rec_mp=0, sigma=1e3)
    base.update(kw)
    return Cueva(45, 38, **base)


def _run(g, n):
    g.step(n)
    g.download()
    return g.prims()


@pytest.mark.parametrize("solver,order", [(7, 2), (5, 3)])
def test_checkpoint_continuation_bit_identical(tmp_path, solver, order):
    a = _ctx(flux_solver=solver, order=order)
    a.kh_init(v0=0.5, a=0.05)
    a.upload()
    a.step(10)
    path = tmp_path / "state.ck"
    a.checkpoint_save(path)
    ref = _run(a, 10)
    h_a, t_a = a.clock()
    b = _ctx(flux_solver=solver, order=order)
    b.checkpoint_load(path)
    assert b.clock() == (10, _t_after(a.dt, 10))
    got = _run(b, 10)
    assert b.clock() == (h_a, t_a)
    for n in ref:
        assert np.array_equal(ref[n], got[n]), n
    a.close(); b.close()


def _t_after(dt, n):
    t = 0.0
    for _ in range(n):
        t = t + dt
    return t


def test_text_backup_continuation_bit_identical(tmp_path):
    a = _ctx()
    a.kh_init(v0=0.5, a=0.05)
    a.upload()
    a.step(6)
    a.download()
    path = tmp_path / "all_variables_0001.dat"
    a.write_all_variables(path)
    h, t = a.clock()
    ref = _run(a, 5)
    b = _ctx()
    b.read_all_variables(path)
    b.upload()
    b.set_clock(h, t)
    got = _run(b, 5)
    for n in ref:
        assert np.array_equal(ref[n], got[n]), n
    a.close(); b.close()


def test_checkpoint_refusals(tmp_path):
    from cueva import Cueva, CuevaError
    a = _ctx()
    a.kh_init(v0=0.5, a=0.05)
    a.upload()
    path = tmp_path / "s.ck"
    a.checkpoint_save(path)
    other = Cueva(46, 38, order=2, flux_solver=7)
    with pytest.raises(CuevaError, match="does not match"):
        other.checkpoint_load(path)
    raw = bytearray(path.read_bytes())
    raw[-9] ^= 0x40
    bad = tmp_path / "bad.ck"
    bad.write_bytes(bytes(raw))
    with pytest.raises(CuevaError, match="checksum"):
        a.checkpoint_load(bad)
    trunc = tmp_path / "trunc.ck"
    trunc.write_bytes(bytes(raw[:-8]))
    with pytest.raises(CuevaError, match="payload"):
        a.checkpoint_load(trunc)
    junk = tmp_path / "junk.ck"
    junk.write_bytes(b"not a checkpoint" * 20)
    with pytest.raises(CuevaError, match="not a version-1"):
        a.checkpoint_load(junk)
    a.close(); other.close()


def test_records_continue_after_checkpoint(tmp_path):
    a = _ctx()
    a.kh_init(v0=0.5, a=0.05)
    a.upload()
    a.step(7)
    path = tmp_path / "s.ck"
    a.checkpoint_save(path)
    b = _ctx()
    b.checkpoint_load(path)
    b.diag_enable(hglb=4)
    b.step(6)
    assert list(b.diagnostics()["h"]) == [8, 12]
    a.close(); b.close()
