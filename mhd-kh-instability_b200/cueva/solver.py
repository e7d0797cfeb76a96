"""Host-side mirror of the reference driver over the C-ABI.

`Cueva` owns Fortran-layout host arrays exactly like the reference's module
arrays -- each field is dimensioned (-6:imax+6, -6:jmax+6) column-major
(threevectors.f95:12-81), stage arrays add a slowest 1:lmax index
(fourvectors.f95:12-170) -- binds them to a context, and exposes the
routines the way main_cueva_code.f95 calls them: ``step`` replaces the body
of the time loop (main_cueva_code.f95:53-328), and ``startconvar``,
``electricvarint``, ``flux_flow``, ``fluxandsource`` (or both at once,
``flux_rhs``), ``varfin``, ``electricfield``, ``con2prim`` mirror the single
routines.
In numpy terms a field is an array of shape (jmax+13, imax+13) (C order,
i fastest) and ``interior(name)`` is its [6:jmax+7, 6:imax+7] view.
"""
import ctypes

import numpy as np

from . import _abi


class Cueva:
    def __init__(self, imax, jmax, order=2, flux_solver=5, rec_mp=0, c2p=1, bc_x=0, bc_y=1, precision=0,
                 device=0, lx=2.0, ly=1.0, lz=1.0, cfl=0.25, sigma=1e3, gamma=4.0 / 3.0, dt=0.0, fma=False,
                 pinned=False, intsum_reset=0, primitive_rec=0):
        self.L = _abi.load(fma)
        self.imax, self.jmax = int(imax), int(jmax)
        self.params = _abi.Params(imax, jmax, order, flux_solver, rec_mp, c2p, bc_x, bc_y, precision, device,
                                  intsum_reset, primitive_rec, lx, ly, lz, cfl, sigma, gamma, dt)
        h = ctypes.c_void_p()
        _abi.check(self.L, self.L.cueva_ctx_create(ctypes.byref(self.params), ctypes.byref(h)))
        self.ctx = h
        self.lmax = self.L.cueva_tableau_stages(self.ctx)
        self.arrays = {}
        self._pinned = []
        self.pinned = pinned
        for name in _abi.PRIM_FIELDS + _abi.CONS_FIELDS:
            self._alloc(name)

    # ---------------------------------------------------------------- arrays
    @property
    def field_shape(self):
        return (self.jmax + 13, self.imax + 13)

    def _alloc(self, name):
        shape = ((self.lmax,) if name in _abi.PER_STAGE else ()) + self.field_shape
        a = np.zeros(shape, dtype=np.float64)
        if self.pinned:
            _abi.check(self.L, self.L.cueva_pin_host(a.ctypes.data_as(ctypes.c_void_p), a.nbytes))
            self._pinned.append(a)
        self.arrays[name] = a
        _abi.check(self.L, self.L.cueva_bind_field(self.ctx, _abi.FIELD_ID[name],
                                                  a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return a

    def array(self, name):
        """Fortran-layout host array bound to the context (allocated on first use)."""
        a = self.arrays.get(name)
        return a if a is not None else self._alloc(name)

    def interior(self, name, l=None):
        a = self.array(name)
        if l is not None:
            a = a[l - 1]
        return a[..., 6:self.jmax + 7, 6:self.imax + 7]

    def set_interior(self, name, values, l=None):
        self.interior(name, l)[...] = values

    def prims(self):
        return {n: self.interior(n).copy() for n in _abi.PRIM_FIELDS}

    # ------------------------------------------------------------- hot path
    @property
    def dt(self):
        return self.L.cueva_dt(self.ctx)

    def kh_init(self, v0=0.5, a=0.01, amp=0.01, width=0.01, kpert=2 * np.pi, phase=0.0, bshear=0.1, rho0=1.0,
                p0=1.0):
        _abi.check(self.L, self.L.cueva_kh_init(self.ctx, v0, a, amp, width, kpert, phase, bshear, rho0, p0))

    def upload(self, groups=_abi.G_PRIMS):
        _abi.check(self.L, self.L.cueva_upload(self.ctx, groups))

    def download(self, groups=_abi.G_PRIMS):
        _abi.check(self.L, self.L.cueva_download(self.ctx, groups))

    def download_async(self, groups=_abi.G_PRIMS):
        """Queues the readback on a second stream; the arrays are complete
        after sync(), and a following upload() waits field by field."""
        _abi.check(self.L, self.L.cueva_download_async(self.ctx, groups))

    def step(self, n=1):
        _abi.check(self.L, self.L.cueva_step(self.ctx, int(n)))

    def sync(self):
        _abi.check(self.L, self.L.cueva_sync(self.ctx))

    def status(self):
        s = ctypes.c_uint32()
        _abi.check(self.L, self.L.cueva_status(self.ctx, ctypes.byref(s)))
        return s.value

    def clear_status(self):
        """Clears the sticky status bits after the caller handled them."""
        _abi.check(self.L, self.L.cueva_clear_status(self.ctx))

    def counters(self):
        c = (ctypes.c_int64 * 3)()
        _abi.check(self.L, self.L.cueva_counters(self.ctx, c))
        return list(c)

    def profile_steps(self, n=1):
        """Advance n steps kernel by kernel (no graph) and return the summed
        device ms and launch counts of the (x-face, y-face, update) kernels."""
        ms = (ctypes.c_double * 3)()
        cnt = (ctypes.c_int32 * 3)()
        _abi.check(self.L, self.L.cueva_profile_steps(self.ctx, n, ms, cnt))
        return list(ms), list(cnt)

    def set_stage_kernel(self, fused):
        """1: one fused kernel per RK stage (the default where it exists: MP5
        and the MC slopes); 0: the y-face and x-face + update kernels.  Both
        give bit-identical results."""
        _abi.check(self.L, self.L.cueva_set_stage_kernel(self.ctx, int(fused)))

    def stage_kernel(self):
        v = ctypes.c_int32()
        _abi.check(self.L, self.L.cueva_get_stage_kernel(self.ctx, ctypes.byref(v)))
        return v.value

    def device_bytes(self):
        """Bytes of device memory the context's field slab holds."""
        v = ctypes.c_uint64()
        _abi.check(self.L, self.L.cueva_device_bytes(self.ctx, ctypes.byref(v)))
        return v.value

    def set_stream(self, stream_ptr):
        _abi.check(self.L, self.L.cueva_set_stream(self.ctx, ctypes.c_void_p(stream_ptr)))

    def set_learned_kernel(self, mode):
        """Learned con2prim: 1 = tcgen05 kernel after the last stage (the
        default once a network is attached), 0 = inside the last stage."""
        _abi.check(self.L, self.L.cueva_set_learned_kernel(self.ctx, int(mode)))

    # ------------------------------------------------------- clock and diagnostics
    def set_clock(self, h, t):
        """Step index h of the last completed step and t_advance (restarts)."""
        _abi.check(self.L, self.L.cueva_set_clock(self.ctx, int(h), float(t)))

    def clock(self):
        h, t = ctypes.c_int64(), ctypes.c_double()
        _abi.check(self.L, self.L.cueva_get_clock(self.ctx, ctypes.byref(h), ctypes.byref(t)))
        return h.value, t.value

    def diag_enable(self, hglb=1, capacity=1024, b0=0.1, lr=3.0, ly=None, delta_rec=None):
        """Device-side records of the writer's diagnostics after every step h
        with h == 1 or h % hglb == 0 (22_writer.f95:821-1019).  Defaults are
        the reference's parameters.f95 values: B0 = 0.1, Lr = 3, Ly = the
        context's y length, delta_rec = a_tm = S_l**(-1/3) * Lr with S_l = 1e3."""
        if ly is None:
            ly = self.params.ly
        if delta_rec is None:
            delta_rec = 1.0e3 ** (-1.0 / 3.0) * lr
        self._diag_cfg = _abi.DiagConfig(int(hglb), int(capacity), b0, lr, ly, delta_rec)
        _abi.check(self.L, self.L.cueva_diag_enable(self.ctx, ctypes.byref(self._diag_cfg)))

    def diag_disable(self):
        _abi.check(self.L, self.L.cueva_diag_enable(self.ctx, None))

    @staticmethod
    def _records_to_dict(recs):
        out = {"h": np.array([r.h for r in recs], dtype=np.int64), "t": np.array([r.t for r in recs])}
        vals = np.array([list(r.v) for r in recs]).reshape(len(recs), _abi.NDIAG)
        for k, name in enumerate(_abi.DIAG_SLOTS):
            out[name] = vals[:, k]
        return out

    def diagnostics(self, max_records=1 << 16):
        """Records appended since the last call, as {slot name: array over records}."""
        buf = (_abi.DiagRecord * max_records)()
        n = ctypes.c_int32()
        _abi.check(self.L, self.L.cueva_diag_read(self.ctx, buf, max_records, ctypes.byref(n)))
        return self._records_to_dict(buf[:n.value])

    def diag_now(self):
        """One record of the current device state (D, tau from startconvar)."""
        r = _abi.DiagRecord()
        _abi.check(self.L, self.L.cueva_diag_now(self.ctx, ctypes.byref(r)))
        return {k: v[0] for k, v in self._records_to_dict([r]).items()}

    # ------------------------------------------------------- checkpoint / restart
    def checkpoint_save(self, path):
        """Binary checkpoint of the device state and the clock."""
        _abi.check(self.L, self.L.cueva_checkpoint_save(self.ctx, str(path).encode()))

    def checkpoint_load(self, path):
        """Replaces the device state and the clock with a checkpoint of the same grid."""
        _abi.check(self.L, self.L.cueva_checkpoint_load(self.ctx, str(path).encode()))

    def write_all_variables(self, path, overwrite=False, nthreads=0):
        """The bound host primitives (ghosts included) as the reference's
        backup file all_variables_NNNN.dat (22_writer.f95:1134-1150)."""
        write_all_variables(path, self.imax, self.jmax, {n: self.array(n) for n in _abi.PRIM_FIELDS},
                            overwrite=overwrite, nthreads=nthreads, lib=self.L)

    def read_all_variables(self, path, nthreads=0):
        """Fills the bound host primitives from a backup file, as
        init_restart does (03_restart_primitive.f95:51-57); upload() next."""
        read_all_variables(path, self.imax, self.jmax, {n: self.array(n) for n in _abi.PRIM_FIELDS},
                           nthreads=nthreads, lib=self.L)

    # ------------------------------------------------------- routine mirrors
    def startconvar(self):
        _abi.check(self.L, self.L.cueva_startconvar(self.ctx))

    def electricvarint(self, l):
        for n in ("Exint", "Eyint", "Ezint", "Jxint", "Jyint", "Jzint"):
            self.array(n)
        _abi.check(self.L, self.L.cueva_electricvarint(self.ctx, int(l)))

    def flux_rhs(self, l):
        for n in _abi.RHS_FIELDS:
            self.array(n)
        _abi.check(self.L, self.L.cueva_flux_rhs(self.ctx, int(l)))

    def flux_flow(self, l):
        """The flux routine alone (lax_flow / hll*_flow / hll*_flow_mpx by
        flux_solver): fills the 28 interface flux arrays of stage l on the
        faces fluxandsource reads (see ``faces``)."""
        for n in _abi.FACE_FIELDS:
            self.array(n)
        _abi.check(self.L, self.L.cueva_flux_flow(self.ctx, int(l)))

    def fluxandsource(self, l):
        """17_fluxandsource.f95 on the bound interface flux arrays of stage l."""
        for n in _abi.FACE_FIELDS + _abi.RHS_FIELDS:
            self.array(n)
        _abi.check(self.L, self.L.cueva_fluxandsource(self.ctx, int(l)))

    def faces(self, name, l):
        """View of an interface flux array on the faces the divergence reads:
        x arrays at i = -1..imax, j = 0..jmax; y arrays at i = 0..imax, j = -1..jmax."""
        a = self.array(name)[l - 1]
        if name in _abi.FACE_X:
            return a[6:self.jmax + 7, 5:self.imax + 7]
        return a[5:self.jmax + 7, 6:self.imax + 7]

    def varfin(self):
        """19_varfin.f95: psi, phi, B, q, D, tau, S += dt * their final sums."""
        for n in _abi.FINSUM_FIELDS:
            self.array(n)
        _abi.check(self.L, self.L.cueva_varfin(self.ctx))

    def electricfield(self):
        """20_electricfield.f95 (IMEX): E += dt * Exfinsum .."""
        for n in _abi.FINSUM_FIELDS:
            self.array(n)
        _abi.check(self.L, self.L.cueva_electricfield(self.ctx))

    def con2prim(self):
        _abi.check(self.L, self.L.cueva_con2prim(self.ctx))

    def close(self):
        if getattr(self, "ctx", None):
            self.L.cueva_ctx_destroy(self.ctx)
            self.ctx = None
        for a in self._pinned:
            self.L.cueva_unpin_host(a.ctypes.data_as(ctypes.c_void_p))
        self._pinned = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_all_variables(path, imax, jmax, arrays=None, nthreads=0, lib=None):
    """Reads a backup file into Fortran-layout arrays (shape (jmax+13,
    imax+13), ghosts included); returns {primitive name: array}.  Host only."""
    L = lib or _abi.load(False)
    if arrays is None:
        arrays = {n: np.zeros((jmax + 13, imax + 13)) for n in _abi.PRIM_FIELDS}
    _abi.check(L, L.cueva_read_all_variables(str(path).encode(), int(imax), int(jmax), _abi.field_table(arrays),
                                             int(nthreads)))
    return arrays


def write_all_variables(path, imax, jmax, arrays, overwrite=False, nthreads=0, lib=None):
    """Writes Fortran-layout primitive arrays as a backup file.  Host only."""
    L = lib or _abi.load(False)
    _abi.check(L, L.cueva_write_all_variables(str(path).encode(), int(imax), int(jmax), _abi.field_table(arrays),
                                              1 if overwrite else 0, int(nthreads)))
