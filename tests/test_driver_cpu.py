"""The C++ driver (mhd-kh-instability_b200/host/cueva_driver.cpp), the
stand-in for the reference's main program over the C-ABI: its command line
and configuration checks, which need no GPU."""
import os
import subprocess

import pytest

from conftest import PKG

DRIVER = os.path.join(PKG, "lib", "cueva_driver")


@pytest.fixture(scope="module")
def driver():
    if not os.path.exists(DRIVER):
        pytest.fail(f"{DRIVER} is missing: build it with `make -C mhd-kh-instability_b200/csrc`")
    return DRIVER


def test_help_lists_the_parameters(driver):
    r = subprocess.run([driver, "--help"], capture_output=True, text=True)
    assert r.returncode == 0
    for key in ("imax", "jmax", "flux_solver", "rec_mp", "conserved_to_primitive", "BOUND", "hglb", "hloc",
                "RESTART", "restart_file", "checkpoint_in"):
        assert key in r.stdout


@pytest.mark.parametrize("text,frag", [("imx = 64\n", "unknown key 'imx'"), ("imax 64\n", "expected key = value"),
                                       ("BOUND = 3\n", "BOUND must be"), ("hmax = 0\n", "hini <= hmax")])
def test_bad_configuration(driver, tmp_path, text, frag):
    cfg = tmp_path / "run.cfg"
    cfg.write_text("! comment line\n" + text)
    r = subprocess.run([driver, str(cfg)], capture_output=True, text=True)
    assert r.returncode == 1 and frag in r.stderr


def test_without_gpu_fails_with_cuda_status(driver, tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    cfg = tmp_path / "run.cfg"
    cfg.write_text("imax = 16\njmax = 8\nhmax = 3\n")
    r = subprocess.run([driver, str(cfg)], capture_output=True, text=True)
    assert r.returncode == 3 and "no CUDA device" in r.stderr
