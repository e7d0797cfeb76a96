"""cueva -- B200 (sm_100a) implementation of the CUEVA per-step hot path.

Python host mirror over the C-ABI of include/cueva.h; the kernels live in
mhd-kh-instability_b200/csrc and are built into mhd-kh-instability_b200/lib.
"""
from ._abi import (CUEVA_ERR_ARG, CUEVA_ERR_CUDA, CUEVA_ERR_PHYSICS, CUEVA_ERR_UNBOUND, CUEVA_OK, FIELDS,
                   G_CONS, G_PRIMS, PRIM_FIELDS, RHS_FIELDS, STAGE_FIELDS, CuevaError, lib_path, load)
from .configs import C1, C2, C3, CONFIGS, TARGET, KHConfig
from .solver import Cueva, read_all_variables, write_all_variables

__all__ = ["Cueva", "read_all_variables", "write_all_variables", "CuevaError", "KHConfig", "C1", "C2", "C3", "TARGET", "CONFIGS", "load", "lib_path",
           "PRIM_FIELDS", "RHS_FIELDS", "STAGE_FIELDS", "FIELDS", "G_PRIMS", "G_CONS", "CUEVA_OK",
           "CUEVA_ERR_ARG", "CUEVA_ERR_CUDA", "CUEVA_ERR_UNBOUND", "CUEVA_ERR_PHYSICS"]
