"""ctypes binding of include/cueva.h (libcueva_b200.so).

The library is built in-tree (mhd-kh-instability_b200/lib); there is no CPU
fallback: if the shared object is missing or no GPU is present the calls fail
loudly with the library's own error message.
"""
import ctypes
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.normpath(os.path.join(_PKG, "..", "lib"))
_LIBS = {}

CUEVA_OK, CUEVA_ERR_ARG, CUEVA_ERR_CUDA, CUEVA_ERR_UNBOUND, CUEVA_ERR_PHYSICS = 0, 1, 2, 3, 4
G_PRIMS, G_CONS = 1, 2

PRIM_FIELDS = ["rho", "p", "vx", "vy", "vz", "psi", "phi", "Ex", "Ey", "Ez", "Bx", "By", "Bz", "q"]
CONS_FIELDS = ["D", "tau", "Sx", "Sy", "Sz", "W"]
STAGE_FIELDS = ["psiint", "phiint", "Exint", "Eyint", "Ezint", "Bxint", "Byint", "Bzint", "qint", "DDint",
                "tauint", "Sxint", "Syint", "Szint", "Jxint", "Jyint", "Jzint", "Exast", "Eyast", "Ezast"]
RHS_FIELDS = ["psiflux", "phiflux", "Exastflux", "Eyastflux", "Ezastflux", "Bxflux", "Byflux", "Bzflux",
              "qflux", "Dflux", "tauflux", "Sxflux", "Syflux", "Szflux", "Exastsour", "Eyastsour", "Ezastsour"]
# stage interface fluxes (the flux routines' outputs read by 17_fluxandsource.f95)
FACE_FIELDS = ["Exlaxpsi", "Eylaxpsi", "Bxlaxphi", "Bylaxphi", "philaxBx", "EzlaxBx", "EzlaxBy", "philaxBy",
               "EylaxBz", "ExlaxBz", "psilaxEx", "BzlaxEx", "BzlaxEy", "psilaxEy", "BylaxEz", "BxlaxEz", "Jxlax",
               "Jylax", "FDxlax", "FDylax", "Ftauxlax", "Ftauylax", "FSxxlax", "FSxylax", "FSxzlax", "FSyxlax",
               "FSyylax", "FSyzlax"]
# x-face arrays (flux through i+1/2); the others are y faces (j+1/2)
FACE_X = {"Exlaxpsi", "Bxlaxphi", "philaxBx", "EzlaxBy", "EylaxBz", "psilaxEx", "BzlaxEy", "BylaxEz", "Jxlax",
          "FDxlax", "Ftauxlax", "FSxxlax", "FSxylax", "FSxzlax"}
# final stage sums (increments of varfin / electricfield)
FINSUM_FIELDS = ["psifinsum", "phifinsum", "Bxfinsum", "Byfinsum", "Bzfinsum", "Exfinsum", "Eyfinsum", "Ezfinsum",
                 "qfinsum", "Dfinsum", "taufinsum", "Sxfinsum", "Syfinsum", "Szfinsum"]
FIELDS = PRIM_FIELDS + CONS_FIELDS + STAGE_FIELDS + RHS_FIELDS + FACE_FIELDS + FINSUM_FIELDS
FIELD_ID = {n: k for k, n in enumerate(FIELDS)}
PER_STAGE = set(STAGE_FIELDS) | set(RHS_FIELDS) | set(FACE_FIELDS)

EXPORTS = ["cueva_ctx_create", "cueva_ctx_destroy", "cueva_last_error", "cueva_set_stream", "cueva_dt",
           "cueva_tableau_stages", "cueva_bind_field", "cueva_pin_host", "cueva_unpin_host", "cueva_upload",
           "cueva_download", "cueva_download_async", "cueva_step", "cueva_sync", "cueva_status", "cueva_counters", "cueva_startconvar",
           "cueva_electricvarint", "cueva_flux_rhs", "cueva_flux_flow", "cueva_fluxandsource", "cueva_varfin", "cueva_electricfield", "cueva_con2prim", "cueva_kh_init", "cueva_profile_steps", "cueva_flux_rhs_noalloc", "cueva_mlp_create",
           "cueva_mlp_destroy", "cueva_mlp_get_params", "cueva_mlp_set_params", "cueva_mlp_synthetic_pairs",
           "cueva_mlp_fit_normalisation", "cueva_mlp_train", "cueva_mlp_gradients", "cueva_mlp_predict",
           "cueva_c2p_batch", "cueva_attach_mlp", "cueva_learned_stats", "cueva_ens_create", "cueva_ens_destroy",
           "cueva_ens_set_stream", "cueva_ens_set_prims", "cueva_ens_get_prims", "cueva_ens_kh_init",
           "cueva_ens_step", "cueva_ens_sync", "cueva_ens_set_shape", "cueva_ens_autotune",
           "cueva_ens_attach_mlp", "cueva_ens_learned_stats", "cueva_set_clock", "cueva_get_clock",
           "cueva_diag_enable", "cueva_diag_read", "cueva_diag_now", "cueva_checkpoint_save",
           "cueva_checkpoint_load", "cueva_read_all_variables", "cueva_write_all_variables",
           "cueva_set_learned_kernel", "cueva_ens_set_learned_kernel", "cueva_clear_status"]
MLP_NPARAM, MLP_NNORM = 8833, 14


class Params(ctypes.Structure):
    _fields_ = [("imax", ctypes.c_int32), ("jmax", ctypes.c_int32), ("order", ctypes.c_int32),
                ("flux_solver", ctypes.c_int32), ("rec_mp", ctypes.c_int32), ("c2p", ctypes.c_int32),
                ("bc_x", ctypes.c_int32), ("bc_y", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("device", ctypes.c_int32), ("intsum_reset", ctypes.c_int32), ("primitive_rec", ctypes.c_int32),
                ("lx", ctypes.c_double), ("ly", ctypes.c_double),
                ("lz", ctypes.c_double), ("cfl", ctypes.c_double), ("sigma", ctypes.c_double),
                ("gamma", ctypes.c_double), ("dt", ctypes.c_double)]


# slots of cueva_diag_record.v (enum cueva_diag_slot); the writer's Fortran unit in brackets
DIAG_SLOTS = ["sum_psi", "sum_phi", "sum_ex", "sum_ey", "sum_ez", "sum_exey", "sum_exez", "sum_eyez",
              "sum_bx", "sum_by", "sum_bz", "sum_bxby", "sum_bxbz", "sum_bybz", "sum_vxvyvz", "sum_bxbybz",
              "sum_vx", "sum_vy", "sum_vz", "sum_vxvy", "sum_vxvz", "sum_vyvz", "sum_q", "sum_p", "sum_rho",
              "ekin_c", "ekin_r", "etot", "efluid_r", "emag", "eint_c", "eint_r", "lorentz", "sum_D",
              "sum_D_med", "max_val_bx", "max_val_phi", "delta_rec_t", "Ez_med", "By_med",
              "max_v", "max_W", "max_lambda_x", "max_lambda_y", "courant"]
DIAG_UNITS = [80, 81, 82, 83, 84, 85, 86, 87, 88, 90, 91, 92, 93, 94, 95, 96, 97, 98, 99,
              200, 201, 202, 203, 204, 205, 206, 207, 208, 209, 210, 211, 212, 213, 214, 215, 216, 217, 67, 68]
NDIAG = len(DIAG_SLOTS)
NDIAG_SUMS = 35


class DiagRecord(ctypes.Structure):
    _fields_ = [("h", ctypes.c_int64), ("t", ctypes.c_double), ("v", ctypes.c_double * NDIAG)]


class DiagConfig(ctypes.Structure):
    _fields_ = [("hglb", ctypes.c_int32), ("capacity", ctypes.c_int32), ("b0", ctypes.c_double),
                ("lr", ctypes.c_double), ("ly", ctypes.c_double), ("delta_rec", ctypes.c_double)]


class CuevaError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"cueva error {code}: {msg}")
        self.code = code


def lib_path(fma=False):
    return os.path.join(LIBDIR, "libcueva_b200_fma.so" if fma else "libcueva_b200.so")


def load(fma=False):
    """Load the C-ABI library: the default build keeps the reference's
    operation order (no FMA contraction); fma=True loads the contracted one."""
    key = bool(fma)
    if key in _LIBS:
        return _LIBS[key]
    path = lib_path(fma)
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: build it with `make -C mhd-kh-instability_b200/csrc`")
    L = ctypes.CDLL(path)
    vp, i32, u32, dbl = ctypes.c_void_p, ctypes.c_int32, ctypes.c_uint32, ctypes.c_double
    L.cueva_ctx_create.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(vp)]
    L.cueva_ctx_destroy.argtypes = [vp]
    L.cueva_last_error.restype = ctypes.c_char_p
    L.cueva_set_stream.argtypes = [vp, vp]
    L.cueva_set_stage_kernel.argtypes = [vp, i32]
    L.cueva_get_stage_kernel.argtypes = [vp, ctypes.POINTER(i32)]
    L.cueva_device_bytes.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64)]
    L.cueva_dt.restype = dbl
    L.cueva_dt.argtypes = [vp]
    L.cueva_tableau_stages.argtypes = [vp]
    L.cueva_bind_field.argtypes = [vp, i32, ctypes.POINTER(ctypes.c_double)]
    L.cueva_pin_host.argtypes = [vp, ctypes.c_uint64]
    L.cueva_unpin_host.argtypes = [vp]
    L.cueva_upload.argtypes = [vp, u32]
    L.cueva_download.argtypes = [vp, u32]
    L.cueva_download_async.argtypes = [vp, u32]
    L.cueva_step.argtypes = [vp, i32]
    L.cueva_sync.argtypes = [vp]
    L.cueva_status.argtypes = [vp, ctypes.POINTER(u32)]
    L.cueva_counters.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
    L.cueva_startconvar.argtypes = [vp]
    L.cueva_electricvarint.argtypes = [vp, i32]
    L.cueva_flux_rhs.argtypes = [vp, i32]
    L.cueva_flux_flow.argtypes = [vp, i32]
    L.cueva_fluxandsource.argtypes = [vp, i32]
    L.cueva_varfin.argtypes = [vp]
    L.cueva_electricfield.argtypes = [vp]
    L.cueva_con2prim.argtypes = [vp]
    L.cueva_kh_init.argtypes = [vp] + [dbl] * 9
    L.cueva_profile_steps.argtypes = [vp, i32, ctypes.POINTER(dbl), ctypes.POINTER(i32)]
    i64, u64, f32p = ctypes.c_int64, ctypes.c_uint64, ctypes.POINTER(ctypes.c_float)
    L.cueva_mlp_create.argtypes = [i32, u64, ctypes.POINTER(vp)]
    L.cueva_mlp_destroy.argtypes = [vp]
    L.cueva_mlp_get_params.argtypes = [vp, f32p, i32]
    L.cueva_mlp_set_params.argtypes = [vp, f32p, i32]
    L.cueva_mlp_synthetic_pairs.argtypes = [i32, i64, u64, dbl, vp, vp, vp]
    L.cueva_mlp_fit_normalisation.argtypes = [vp, vp, vp, i64]
    L.cueva_mlp_train.argtypes = [vp, vp, vp, i64, i32, i32, ctypes.c_float, u64, f32p]
    L.cueva_mlp_gradients.argtypes = [vp, vp, vp, i32, f32p, f32p]
    L.cueva_mlp_predict.argtypes = [vp, vp, i64, vp, i32]
    L.cueva_c2p_batch.argtypes = [i32, i32, vp, dbl, dbl, vp, vp, vp, i64, vp, vp]
    L.cueva_attach_mlp.argtypes = [vp, vp]
    L.cueva_learned_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
    L.cueva_ens_create.argtypes = [ctypes.POINTER(Params), i32, ctypes.POINTER(vp)]
    L.cueva_ens_destroy.argtypes = [vp]
    L.cueva_ens_set_stream.argtypes = [vp, vp]
    L.cueva_ens_set_prims.argtypes = [vp, i32, ctypes.POINTER(dbl)]
    L.cueva_ens_get_prims.argtypes = [vp, i32, ctypes.POINTER(dbl)]
    L.cueva_ens_kh_init.argtypes = [vp, i32] + [dbl] * 9
    L.cueva_ens_step.argtypes = [vp, i32]
    L.cueva_ens_sync.argtypes = [vp, ctypes.POINTER(u32)]
    L.cueva_ens_set_shape.argtypes = [vp, i32, i32]
    L.cueva_ens_autotune.argtypes = [vp, ctypes.POINTER(i32), ctypes.POINTER(i32), ctypes.POINTER(dbl)]
    L.cueva_ens_attach_mlp.argtypes = [vp, vp]
    L.cueva_ens_learned_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
    L.cueva_set_clock.argtypes = [vp, i64, dbl]
    L.cueva_get_clock.argtypes = [vp, ctypes.POINTER(i64), ctypes.POINTER(dbl)]
    L.cueva_diag_enable.argtypes = [vp, ctypes.POINTER(DiagConfig)]
    L.cueva_diag_read.argtypes = [vp, ctypes.POINTER(DiagRecord), i32, ctypes.POINTER(i32)]
    L.cueva_diag_now.argtypes = [vp, ctypes.POINTER(DiagRecord)]
    L.cueva_set_learned_kernel.argtypes = [vp, i32]
    L.cueva_clear_status.argtypes = [vp]
    L.cueva_ens_set_learned_kernel.argtypes = [vp, i32]
    L.cueva_checkpoint_save.argtypes = [vp, ctypes.c_char_p]
    L.cueva_checkpoint_load.argtypes = [vp, ctypes.c_char_p]
    dpp = ctypes.POINTER(ctypes.POINTER(dbl))
    L.cueva_read_all_variables.argtypes = [ctypes.c_char_p, i32, i32, dpp, i32]
    L.cueva_write_all_variables.argtypes = [ctypes.c_char_p, i32, i32, dpp, i32, i32]
    L.cueva_flux_rhs_noalloc.argtypes = [ctypes.POINTER(Params), vp, vp, vp, vp, i32, ctypes.c_int64, vp,
                                         ctypes.POINTER(u32)]
    _LIBS[key] = L
    return L


def check(L, rc):
    if rc != CUEVA_OK:
        raise CuevaError(rc, L.cueva_last_error().decode())
    return rc


def field_table(arrays):
    """ctypes table of pointers indexed by enum cueva_field for the 14
    primitive arrays in `arrays` (name -> Fortran-layout float64 array)."""
    tab = (ctypes.POINTER(ctypes.c_double) * len(PRIM_FIELDS))()
    for k, n in enumerate(PRIM_FIELDS):
        a = arrays[n]
        if a.dtype != "float64" or not a.flags["C_CONTIGUOUS"]:
            raise ValueError(f"{n}: a C-contiguous float64 array is required")
        tab[k] = a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    return tab
