"""C-ABI checks that need no GPU: the in-tree libraries load, export every
entry point include/cueva.h declares, agree with the header's field table,
and reject bad configurations with the documented error classes."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "cueva.h")


def _declared():
    text = open(HEADER).read()
    return re.findall(r"^(?:int32_t|double|const char\*)\s+(cueva_\w+)\s*\(", text, re.M)


def _field_enum():
    text = open(HEADER).read()
    body = text[text.index("enum cueva_field {"):text.index("CUEVA_NFIELDS")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    return re.findall(r"CUEVA_(\w+)", body)


@pytest.mark.parametrize("fma", [False, True])
def test_library_exports_every_declared_symbol(fma):
    import cueva
    L = cueva.load(fma)
    names = _declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), f"{n} declared in cueva.h but not exported by {cueva.lib_path(fma)}"


def test_python_field_table_matches_header():
    from cueva import _abi
    enum = _field_enum()
    assert [e.lower() for e in enum] == [f.lower() for f in _abi.FIELDS]


def test_fortran_module_field_ids_match_header():
    """fortran/cueva_gpu.f90 names every field id of enum cueva_field with
    the same value (the Fortran side binds its arrays by these numbers)."""
    text = open(os.path.join(ROOT, "mhd-kh-instability_b200", "fortran", "cueva_gpu.f90")).read()
    ids = {m.group(1).upper(): int(m.group(2)) for m in re.finditer(r"CUEVA_(\w+)\s*=\s*(\d+)", text)}
    for k, name in enumerate(_field_enum()):
        assert ids.get(name.upper()) == k, (name, ids.get(name.upper()), k)


def test_params_struct_layout():
    from cueva import _abi
    # 12 int32 then 7 doubles, as declared in cueva.h
    assert ctypes.sizeof(_abi.Params) == 12 * 4 + 7 * 8
    assert _abi.Params.lx.offset == 48


def _create(**kw):
    import cueva
    from cueva import _abi
    L = cueva.load(False)
    base = dict(imax=64, jmax=32, order=2, flux_solver=5, rec_mp=0, c2p=1, bc_x=0, bc_y=1, precision=0,
                device=0, intsum_reset=0, primitive_rec=0, lx=2.0, ly=1.0, lz=1.0, cfl=0.25, sigma=1e3,
                gamma=4.0 / 3.0, dt=0.0)
    base.update(kw)
    p = _abi.Params(**base)
    h = ctypes.c_void_p()
    rc = L.cueva_ctx_create(ctypes.byref(p), ctypes.byref(h))
    msg = L.cueva_last_error().decode()
    if rc == 0:
        L.cueva_ctx_destroy(h)
    return rc, msg


@pytest.mark.parametrize("kw,frag", [
    (dict(imax=4), "imax"), (dict(flux_solver=8), "flux_solver"), (dict(rec_mp=5), "rec_mp"),
    (dict(c2p=7), "c2p"), (dict(bc_x=2), "bc_x"), (dict(order=7), "order"), (dict(precision=3), "precision"),
    (dict(intsum_reset=2), "intsum_reset"), (dict(primitive_rec=3), "primitive_rec")])
def test_bad_configuration_rejected(kw, frag):
    rc, msg = _create(**kw)
    assert rc == 1 and frag.split("_")[0] in msg.lower().replace(" ", "_")


def test_create_without_gpu_fails_loudly():
    import torch
    rc, msg = _create()
    if torch.cuda.is_available():
        assert rc == 0
    else:
        assert rc == 2 and "device" in msg


def test_diag_record_table_matches_header():
    """The Python slot table follows enum cueva_diag_slot, and its writer
    units are the bracketed units of the header comments."""
    from cueva import _abi
    text = open(HEADER).read()
    body = text[text.index("enum cueva_diag_slot {"):text.index("CUEVA_NDIAG\n")]
    slots = re.findall(r"^\s*CUEVA_DG_(\w+)", body, re.M)
    assert len(slots) == _abi.NDIAG == len(_abi.DIAG_SLOTS)
    units = [int(u) for u in re.findall(r"/\* \[(\d+)\]", body)]
    assert units == _abi.DIAG_UNITS
    assert ctypes.sizeof(_abi.DiagRecord) == 16 + 8 * _abi.NDIAG
    assert ctypes.sizeof(_abi.DiagConfig) == 8 + 4 * 8
