"""GPU: the C++ driver end to end.  A run writes the writer's time series
(data_global/, units 67, 68, 80-99, 200-217) and backups
(data_restart/all_variables_NNNN.dat) that equal the library's own records
and state bit for bit, follows the oracle within the parity bar, and a
restart from its backup or from a binary checkpoint reproduces the
uninterrupted run exactly."""
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG, rel_l1_field

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(PKG, "lib", "cueva_driver")
BASE = dict(imax=64, jmax=32, order=2, flux_solver=7, rec_mp=0, sigma=1e3, hglb=5, hloc=10, kh_a=0.05)


def _run(tmp, name, **kw):
    cfg = dict(BASE)
    cfg.update(kw)
    out = tmp / name
    cfg["output_dir"] = str(out)
    path = tmp / f"{name}.cfg"
    path.write_text("".join(f"{k} = {v}\n" for k, v in cfg.items()))
    r = subprocess.run([DRIVER, str(path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return out


def _series(out, fname):
    return np.loadtxt(out / "data_global" / fname, ndmin=2)


def _python_run(steps):
    from cueva import Cueva
    g = Cueva(64, 32, order=2, flux_solver=7, rec_mp=0, sigma=1e3)
    g.kh_init(v0=0.5, a=0.05)
    g.upload()
    g.diag_enable(hglb=5)
    states = {}
    for h in range(1, steps + 1):
        g.step(1)
        if h % 10 == 0:
            g.download()
            states[h] = g.prims()
    recs = g.diagnostics()
    g.close()
    return recs, states


def test_driver_series_and_backups_match_library(tmp_path):
    from cueva import _abi, read_all_variables
    out = _run(tmp_path, "A", hmax=21)
    recs, states = _python_run(20)
    assert list(recs["h"]) == [1, 5, 10, 15, 20]
    units = dict(zip(_abi.DIAG_UNITS, _abi.DIAG_SLOTS))
    files = {80: "2d_data_psi_integral_vol.dat", 208: "2d_data_etot_integral_vol.dat",
             212: "2d_data_eint_r_integral_vol.dat", 216: "2d_data_bx_max_val.dat", 67: "delta_rec_t_2D.dat",
             68: "rate_rec_ez_2D.dat", 213: "2d_data_lorentz_integral_vol.dat"}
    for unit, fname in files.items():
        s = _series(out, fname)
        assert list(s[:, 0]) == [1, 5, 10, 15, 20]
        assert np.array_equal(s[:, 1], recs["t"]), fname
        assert np.array_equal(s[:, 2], recs[units[unit]]), fname
    assert len(os.listdir(out / "data_global")) == 40   # 39 writer units + the Courant check
    for hb in (1, 2):
        g = read_all_variables(out / "data_restart" / f"all_variables_{hb:04d}.dat", 64, 32)
        for n, ref in states[10 * hb].items():
            assert np.array_equal(g[n][6:6 + 33, 6:6 + 65], ref), (hb, n)
        # ghosts: x copy (BOUND 6), y periodic node duplicates
        rho = g["rho"]
        assert np.array_equal(rho[6:39, 0], rho[6:39, 6]) and np.array_equal(rho[6:39, -1], rho[6:39, 6 + 64])
        assert np.array_equal(rho[0, 6:71], rho[6 + 32 - 6, 6:71]) and np.array_equal(rho[38 + 6, 6:71], rho[6 + 6, 6:71])


def test_driver_follows_the_oracle(tmp_path, oracle_mod):
    from cueva import read_all_variables
    out = _run(tmp_path, "O", hmax=21, hloc=20)
    g = read_all_variables(out / "data_restart" / "all_variables_0001.dat", 64, 32)
    oracle_mod.set_libm_seed(0)
    o = oracle_mod.Oracle(64, 32, order=2, flux_solver=7, rec_mp=0, sigma=1e3)
    o.set_prims(oracle_mod.kh_init(64, 32, v0=0.5, a=0.05))
    assert o.step(20) == 0
    ref = o.get_prims()
    for n, r in ref.items():
        got = g[n][6:39, 6:71]
        assert rel_l1_field(n, got, r, ref) <= 1e-9, n


def test_driver_restart_from_backup_and_checkpoint(tmp_path):
    a = _run(tmp_path, "A", hmax=21)
    b = _run(tmp_path, "B", hmax=21, hini=11, RESTART=1,
             restart_file=str(a / "data_restart" / "all_variables_0001.dat"))
    fa = (a / "data_restart" / "all_variables_0002.dat").read_bytes()
    assert (b / "data_restart" / "all_variables_0002.dat").read_bytes() == fa
    sa, sb = _series(a, "2d_data_etot_integral_vol.dat"), _series(b, "2d_data_etot_integral_vol.dat")
    assert list(sb[:, 0]) == [15, 20] and np.array_equal(sa[3:, 2], sb[:, 2])
    ck = tmp_path / "c.ck"
    _run(tmp_path, "C", hmax=11, checkpoint_out=str(ck))
    d = _run(tmp_path, "D", hmax=21, checkpoint_in=str(ck))
    assert (d / "data_restart" / "all_variables_0002.dat").read_bytes() == fa
    sd = _series(d, "2d_data_etot_integral_vol.dat")
    assert np.array_equal(sa[3:], sd)   # the checkpoint carries the clock: t identical too
