"""B200 dynamical core of UoM-maul1609/dynamical-cloud-model: Python binding.

A thin ctypes layer over libdcm_b200.so (include/dcm.h).  The functions keep
the names, argument meaning and in/out behaviour of the reference Fortran
routines they replace -- bicgstab, sources, advance_momentum, mpdata_3d,
mpdata_vec_3d, first_order_upstream_3d, adv_ref_state, mpdata_3d_add,
horizontal_means, divergence_calc, advance_scalar_fields_3d and the halo
exchanges -- with the MPI arguments dropped (one rank, whole domain on one
GPU).  Arrays are numpy float64 arrays of shape (kp+2, jp+2, ip+2) in Fortran
order, i.e. the reference's a(0:kp+1, 0:jp+1, 0:ip+1); arguments the
reference declares intent(inout) are updated in place.

Errors: a non-zero status raises DCMError carrying the status, the same
conditions on which the reference STOPs.  There is no CPU fallback: if the
CUDA library cannot be loaded, importing the binding raises.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libdcm_b200.so")

DCM_OK, DCM_E_NOCONV, DCM_E_BREAKDOWN, DCM_E_NONFINITE, DCM_E_CUDA = 0, 1, 2, 3, 4
DCM_E_TIMEOUT, DCM_E_DECOMP, DCM_E_ARG, DCM_E_UNSUPPORTED, DCM_E_IO = 5, 6, 7, 8, 9

_dp = C.POINTER(C.c_double)


class DCMError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("dcm status %d: %s" % (status, msg))
        self.status = status


class _Grid(C.Structure):
    _fields_ = [("ip", C.c_int), ("jp", C.c_int), ("kp", C.c_int)] + [
        (n, _dp) for n in ("dx", "dxn", "dy", "dyn", "dz", "dzn", "rhoa", "rhoan", "theta",
                           "thetan", "xg", "yg", "zg")]


class _Forcing(C.Structure):
    _fields_ = [("damping_layer", C.c_int), ("forcing", C.c_int), ("divergence", C.c_int),
                ("dampfacn", _dp), ("dampfac", _dp), ("u_force", _dp), ("v_force", _dp),
                ("w_subs", _dp), ("forcing_tau", C.c_double)]


class _Config(C.Structure):
    _fields_ = [("dt", C.c_double), ("ptol", C.c_double), ("advection_scheme", C.c_int),
                ("kord", C.c_int), ("monotone", C.c_int), ("limiter", C.c_int),
                ("itmax", C.c_int), ("moisture", C.c_int), ("nq", C.c_int), ("ncat", C.c_int),
                ("c_s", C.POINTER(C.c_int)), ("c_e", C.POINTER(C.c_int)),
                ("thbase", C.c_double), ("thtop", C.c_double), ("precision", C.c_int),
                ("inner_tol", C.c_double), ("forcing", _Forcing), ("viscous", C.c_int),
                ("lamsq", _dp), ("z0", C.c_double), ("z0th", C.c_double),
                ("precond", C.c_int), ("precond_lo", C.c_double)]


class _Fields(C.Structure):
    _fields_ = [(n, _dp) for n in ("u", "v", "w", "zu", "zv", "zw", "tu", "tv", "tw", "th", "p",
                                   "su", "sv", "sw", "psrc", "div", "sth", "q", "sq", "ubar",
                                   "vbar", "wbar", "thbar", "qbar")]


class EnsembleStats(C.Structure):
    _fields_ = [("steps", C.c_int), ("iters_total", C.c_longlong), ("iters_max_last", C.c_int),
                ("ms_total", C.c_double)]


class StepStats(C.Structure):
    _fields_ = [("steps", C.c_int), ("iters_last", C.c_int), ("iters_total", C.c_longlong),
                ("err_last", C.c_double), ("ms_total", C.c_double),
                ("updates_last", C.c_int), ("restarts_last", C.c_int)]


_lib = None


def library():
    """Load libdcm_b200.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise OSError("libdcm_b200.so is not built; run build.py (sm_100a)")
        lib = C.CDLL(LIBPATH)
        P = C.c_void_p
        sig = {
            "dcm_create": [C.POINTER(_Grid), C.c_int, C.POINTER(P)],
            "dcm_destroy": [P],
            "dcm_status_string": [C.c_int],
            "dcm_last_error": [P],
            "dcm_check_decomposition": [C.POINTER(C.c_int)],
            "dcm_bicgstab": [P, _dp, _dp, _dp, C.c_double, C.c_int, C.c_int,
                             C.POINTER(C.c_int), _dp],
            "dcm_sources": [P, C.POINTER(_Forcing)] + [_dp] * 16,
            "dcm_advance_momentum": [P, C.c_double] + [_dp] * 10,
            "dcm_first_order_upstream_3d": [P, C.c_double, _dp, _dp, _dp, _dp, C.c_int],
            "dcm_mpdata_3d": [P, C.c_double, _dp, _dp, _dp, _dp, _dp, _dp, C.c_int, C.c_int,
                              C.c_int, C.c_int],
            "dcm_mpdata_vec_3d": [P, C.c_double, _dp, _dp, _dp, _dp, C.c_int, _dp, _dp,
                                  C.c_int, C.c_int, C.c_int, C.c_int],
            "dcm_adv_ref_state": [P, C.c_double, _dp, _dp, _dp],
            "dcm_mpdata_3d_add": [P, C.c_double, _dp, _dp, _dp, _dp, _dp, _dp, _dp, C.c_int,
                                  C.c_int, C.c_int, C.c_int],
            "dcm_horizontal_means": [P, C.c_int, C.c_int] + [_dp] * 10,
            "dcm_divergence_calc": [P, _dp, _dp, _dp, _dp],
            "dcm_advance_scalar_fields_3d": [P, C.c_double, _dp, _dp, _dp, _dp, C.c_int,
                                             C.c_int],
            "dcm_exchange_full": [P, _dp, C.c_double, C.c_double],
            "dcm_exchange_along_dim": [P, _dp, C.c_double, C.c_double],
            "dcm_exchange_along_dim_wo": [P, _dp],
            "dcm_exchange_full_wo": [P, _dp],
            "dcm_calculate_subgrid_3d": [P, _dp, C.c_double, C.c_double] + [_dp] * 7 +
                                        [C.c_int] + [_dp] * 16 + [C.c_int],
            "dcm_state_upload": [P, C.POINTER(_Config), C.POINTER(_Fields)],
            "dcm_driver_start": [P],
            "dcm_step": [P, C.c_int, C.POINTER(StepStats)],
            "dcm_state_download": [P, C.POINTER(_Fields)],
            "dcm_horizontal_means_noalloc": [C.c_int, C.c_int, C.c_int, P, P, P, P, P, P],
            "dcm_mpdata_vec_1d": [C.c_int] * 5 + [_dp, C.POINTER(C.c_int)] + [_dp] * 4 +
                                 [C.c_int, _dp, _dp, C.c_int, C.c_int, C.c_int],
            "dcm_mpdata_vec_1d_device": [C.c_int] * 5 + [P, P] + [P] * 4 +
                                        [C.c_int, P, P, C.c_int, C.c_int, C.c_int, P],
            "dcm_profile_enable": [P, C.c_int],
            "dcm_profile_read": [P, _dp, C.POINTER(C.c_longlong), C.c_int],
            "dcm_solver_graphs": [P, C.c_int],
            "dcm_solver_graph_info": [P, C.POINTER(C.c_int)],
            "dcm_solver_limits": [P, C.c_int, C.c_double],
            "dcm_set_mpdata_shape": [P, C.c_int, C.c_int],
            "dcm_set_small_solver": [P, C.c_int],
            "dcm_tune": [P, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                         C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)],
            "dcm_set_launch_shape": [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int],
            "dcm_ensemble_create": [C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_void_p)],
            "dcm_ensemble_destroy": [P],
            "dcm_ensemble_member": [P, C.c_int, C.POINTER(C.c_void_p)],
            "dcm_ensemble_step": [P, C.c_int, C.POINTER(EnsembleStats)],
            "dcm_ensemble_last_error": [P],
            "dcm_output_open": [P, C.c_char_p, _dp, _dp, _dp, _dp, C.c_int, C.c_char_p, C.c_int,
                                C.POINTER(C.c_void_p)],
            "dcm_output_write": [P, C.c_double],
            "dcm_output_flush": [P],
            "dcm_output_close": [P],
            "dcm_output_last_error": [P],
        }
        for name, args in sig.items():
            f = getattr(lib, name)
            f.argtypes = args
            f.restype = C.c_char_p if name in ("dcm_status_string", "dcm_last_error",
                                               "dcm_ensemble_last_error",
                                               "dcm_output_last_error") else C.c_int
        _lib = lib
    return _lib


EXPORTS = ("dcm_create", "dcm_destroy", "dcm_status_string", "dcm_last_error",
           "dcm_check_decomposition", "dcm_bicgstab", "dcm_sources", "dcm_advance_momentum",
           "dcm_first_order_upstream_3d", "dcm_mpdata_3d", "dcm_mpdata_vec_3d",
           "dcm_adv_ref_state", "dcm_mpdata_3d_add", "dcm_horizontal_means",
           "dcm_divergence_calc", "dcm_advance_scalar_fields_3d", "dcm_exchange_full",
           "dcm_exchange_along_dim", "dcm_exchange_along_dim_wo", "dcm_state_upload",
           "dcm_driver_start", "dcm_step", "dcm_state_download", "dcm_profile_enable",
           "dcm_profile_read", "dcm_horizontal_means_noalloc", "dcm_solver_graphs",
           "dcm_solver_graph_info", "dcm_solver_limits", "dcm_set_mpdata_shape",
           "dcm_set_small_solver", "dcm_tune",
           "dcm_set_launch_shape", "dcm_ensemble_create", "dcm_ensemble_destroy", "dcm_ensemble_member",
           "dcm_ensemble_step", "dcm_ensemble_last_error", "dcm_exchange_full_wo",
           "dcm_calculate_subgrid_3d", "dcm_output_open", "dcm_output_write",
           "dcm_output_flush", "dcm_output_close", "dcm_output_last_error",
           "dcm_mpdata_vec_1d", "dcm_mpdata_vec_1d_device")

PROF_CLASSES = ("setup", "jacobi", "matvec", "update", "post", "means", "sources", "rhs",
                "adv_ref", "mp_shift", "upwind", "antidiff", "beta", "limit", "restore",
                "momentum", "other")


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if a.dtype != np.float64 or not (a.flags.f_contiguous or a.ndim == 1 or
                                         a.flags.c_contiguous):
            raise TypeError("expected a contiguous float64 array")
        return a.ctypes.data_as(_dp)
    raise TypeError("expected a numpy array")


def _field(a, shape):
    if not isinstance(a, np.ndarray) or a.dtype != np.float64 or a.shape != shape or \
            not a.flags.f_contiguous:
        raise TypeError("expected a Fortran-ordered float64 array of shape %s" % (shape,))
    return a.ctypes.data_as(_dp)


def _grid_struct(grid):
    keep = [np.ascontiguousarray(getattr(grid, n), dtype=np.float64)
            for n in ("dx", "dxn", "dy", "dyn", "dz", "dzn", "rhoa", "rhoan", "theta", "thetan",
                      "x", "y", "z")]
    return keep, _Grid(grid.ip, grid.jp, grid.kp, *[a.ctypes.data_as(_dp) for a in keep])


def check_decomposition(dims):
    """mpi_cart_initialise check: only a 1 x 1 x 1 process grid runs here."""
    d = (C.c_int * 3)(*dims)
    st = library().dcm_check_decomposition(d)
    if st:
        raise DCMError(st, library().dcm_status_string(st).decode())


def mpdata_vec_1d_columns(dt, nsub, dz, dzn, rhoa, rhoan, w, psi, kord=1, monotone=False,
                          neumann=0, l_h=1, r_h=1):
    """The PAMM sedimentation transport of ncol columns on the GPU, in place
    on psi (dcm_mpdata_vec_1d: mpdata_vec_1d, pamm/sfvt/advection_1d.F90:463-778,
    nsub[c] passes of dt[c]/nsub[c]).  w: (ncol, kp+l_h+r_h), each row
    w(-l_h+1:kp+r_h); psi: (ncol, nq, kp+2 r_h) C-contiguous, each column's
    psi_in(-r_h+1:kp+r_h, 1:nq); dz, dzn, rhoa, rhoan: (kp+l_h+r_h,) shared or
    (ncol, kp+l_h+r_h) per column.  dt and nsub: scalars or one per column
    (nsub None: one pass)."""
    if not (isinstance(psi, np.ndarray) and psi.dtype == np.float64 and psi.ndim == 3 and
            psi.flags.c_contiguous):
        raise TypeError("psi: a C-contiguous float64 array (ncol, nq, kp+2 r_h)")
    ncol, nq, npsi = psi.shape
    kp = npsi - 2 * r_h
    nw = kp + l_h + r_h
    w = np.ascontiguousarray(w, dtype=np.float64)
    if w.shape != (ncol, nw):
        raise TypeError("w: shape (ncol, kp+l_h+r_h)")
    met = [np.ascontiguousarray(a, dtype=np.float64) for a in (dz, dzn, rhoa, rhoan)]
    stride = nw if met[0].ndim == 2 else 0
    for a in met:
        if a.shape != ((ncol, nw) if stride else (nw,)):
            raise TypeError("dz, dzn, rhoa, rhoan: shape (kp+l_h+r_h,) or (ncol, kp+l_h+r_h)")
    dt = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, dtype=np.float64), (ncol,)))
    ns = None if nsub is None else np.ascontiguousarray(
        np.broadcast_to(np.asarray(nsub, dtype=np.int32), (ncol,)))
    st = library().dcm_mpdata_vec_1d(
        ncol, kp, nq, l_h, r_h, _ptr(dt),
        None if ns is None else ns.ctypes.data_as(C.POINTER(C.c_int)), *[_ptr(a) for a in met],
        stride, _ptr(w), _ptr(psi), int(kord), int(bool(monotone)), int(neumann))
    if st:
        raise DCMError(st, library().dcm_status_string(st).decode())
    return psi


class DynamicalCore:
    """One device handle for one grid (the module state of d_solver lives
    here: the stencil coefficients and the bicgstab first-call flag)."""

    def __init__(self, grid, device=0, _handle=None):
        self.lib = library()
        self.grid = grid
        self.shape = (grid.kp + 2, grid.jp + 2, grid.ip + 2)
        self._state_keep = None
        self._owned = _handle is None
        if _handle is not None:  # a member handle owned by an Ensemble
            self.h = _handle
            return
        self._keep, g = _grid_struct(grid)
        h = C.c_void_p()
        st = self.lib.dcm_create(C.byref(g), device, C.byref(h))
        if st:
            raise DCMError(st, self.lib.dcm_status_string(st).decode())
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            if self._owned:
                self.lib.dcm_destroy(self.h)
            self.h = None

    def tune(self, precision=1, use_cache=True):
        """Autotune the solver launch shape for this grid (dcm_tune); returns
        (warps per sweep block, warp tasks per warp, marching depth, fused,
        levels per lane)."""
        by, tasks, depth, fuse, vec = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_int()
        self._check(self.lib.dcm_tune(self.h, int(precision), int(bool(use_cache)), C.byref(by),
                                      C.byref(tasks), C.byref(depth), C.byref(fuse),
                                      C.byref(vec)))
        return by.value, tasks.value, depth.value, fuse.value, vec.value

    def set_launch_shape(self, precision, by=8, tasks=0, depth=None, fuse=None, vec=None):
        """Set the solver launch shape of one precision (dcm_set_launch_shape).
        fuse: 0 separate sweeps, 1 fused preconditioner, 2 fused with phase
        C's matvec (FP32); vec: levels per lane of the separate kernels (FP32
        4 or 2, FP64 2)."""
        if fuse is None:
            fuse = 1 if precision == 1 else 0
        if depth is None:
            depth = 1 if precision == 1 else 4
        if vec is None:
            vec = 4 if precision == 1 else 2
        self._check(self.lib.dcm_set_launch_shape(self.h, int(precision), int(by), int(tasks),
                                                  int(depth), int(fuse), int(vec)))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st:
            msg = self.lib.dcm_last_error(self.h)
            raise DCMError(st, (msg or b"").decode() or
                           self.lib.dcm_status_string(st).decode())

    def F(self, a):
        return _field(a, self.shape)

    # ---- dynamics.f90 ---------------------------------------------------------
    def bicgstab(self, x, b, sw, tol, test_solver=False, itmax=9999):
        """bicgstab (dynamics.f90:293-444); x, b updated in place.
        Returns (iterations, final relative residual)."""
        it = C.c_int(0)
        err = C.c_double(0.0)
        st = self.lib.dcm_bicgstab(self.h, self.F(x), self.F(b), self.F(sw), float(tol),
                                   int(bool(test_solver)), int(itmax), C.byref(it),
                                   C.byref(err))
        self._check(st)
        return it.value, err.value

    def sources(self, ubar, vbar, wbar, thbar, zu, zv, zw, u, v, w, th, su, sv, sw, sth, rhs,
                forcing=None):
        """sources (dynamics.f90:639-1000), viscous = .false.; su, sv, sw,
        sth, rhs updated in place.  forcing: dict with damping_layer,
        forcing, divergence, dampfacn, dampfac, u_force, v_force, w_subs,
        forcing_tau (all optional)."""
        fs, keep = self._forcing(forcing)
        st = self.lib.dcm_sources(self.h, C.byref(fs) if fs is not None else None,
                                  _ptr(ubar), _ptr(vbar), _ptr(wbar), _ptr(thbar),
                                  *[self.F(a) if a is not None else None for a in (zu, zv, zw)],
                                  self.F(u), self.F(v), self.F(w), self.F(th), self.F(su),
                                  self.F(sv), self.F(sw), self.F(sth), self.F(rhs))
        self._check(st)

    def _forcing(self, f):
        if not f:
            return None, None
        keep = {}
        fs = _Forcing()
        fs.damping_layer = int(f.get("damping_layer", 0))
        fs.forcing = int(f.get("forcing", 0))
        fs.divergence = int(f.get("divergence", 0))
        fs.forcing_tau = float(f.get("forcing_tau", 1.0))
        for n in ("dampfacn", "dampfac", "u_force", "v_force", "w_subs"):
            a = f.get(n)
            if a is not None:
                a = np.ascontiguousarray(a, dtype=np.float64)
                keep[n] = a
                setattr(fs, n, a.ctypes.data_as(_dp))
        return fs, keep

    def advance_momentum(self, dt, u, v, w, zu, zv, zw, su, sv, sw, p):
        """advance_momentum (dynamics.f90:1019-1099); u, v, w in place."""
        self._check(self.lib.dcm_advance_momentum(
            self.h, float(dt), *[self.F(a) for a in (u, v, w, zu, zv, zw, su, sv, sw, p)]))

    # ---- pamm/sfvt/advection_3d.F90 -------------------------------------------
    def first_order_upstream_3d(self, dt, u, v, w, psi, neumann=0):
        self._check(self.lib.dcm_first_order_upstream_3d(
            self.h, float(dt), self.F(u), self.F(v), self.F(w), self.F(psi), int(neumann)))

    def mpdata_3d(self, dt, u, v, w, psi, lbc, ubc, kord, monotone, neumann=0, limiter=0):
        """mpdata_3d; psi in place.  Returns the updated (lbc, ubc)."""
        lb = C.c_double(lbc)
        ub = C.c_double(ubc)
        self._check(self.lib.dcm_mpdata_3d(self.h, float(dt), self.F(u), self.F(v), self.F(w),
                                           self.F(psi), C.byref(lb), C.byref(ub), int(kord),
                                           int(bool(monotone)), int(neumann), int(limiter)))
        return lb.value, ub.value

    def mpdata_vec_3d(self, dt, u, v, w, psi, lbc, ubc, kord, monotone, neumann=0, limiter=0):
        """mpdata_vec_3d; psi is (nq, kp+2, jp+2, ip+2) with each field in
        Fortran order (Fortran psi(:,:,:,1:nq)); lbc/ubc float64 arrays of
        length nq updated in place."""
        if psi.dtype != np.float64 or psi.ndim != 4 or psi.shape[1:] != self.shape:
            raise TypeError("psi must be (nq, kp+2, jp+2, ip+2) float64")
        if not all(psi[q].flags.f_contiguous for q in range(psi.shape[0])) or \
                not _stacked(psi):
            raise TypeError("psi fields must be consecutive Fortran-ordered blocks")
        nq = psi.shape[0]
        self._check(self.lib.dcm_mpdata_vec_3d(self.h, float(dt), self.F(u), self.F(v),
                                               self.F(w), psi.ctypes.data_as(_dp), nq,
                                               _ptr(lbc), _ptr(ubc), int(kord),
                                               int(bool(monotone)), int(neumann), int(limiter)))

    def adv_ref_state(self, dt, w, psi, psi_ref):
        self._check(self.lib.dcm_adv_ref_state(self.h, float(dt), self.F(w), self.F(psi),
                                               _ptr(np.ascontiguousarray(psi_ref))))

    def mpdata_3d_add(self, dt, u, v, w, psi, psi_1d, lbc, ubc, kord, monotone, neumann=0,
                      limiter=0):
        lb = C.c_double(lbc)
        ub = C.c_double(ubc)
        prof = np.ascontiguousarray(psi_1d, dtype=np.float64)
        self._check(self.lib.dcm_mpdata_3d_add(self.h, float(dt), self.F(u), self.F(v),
                                               self.F(w), self.F(psi), _ptr(prof), C.byref(lb),
                                               C.byref(ub), int(kord), int(bool(monotone)),
                                               int(neumann), int(limiter)))
        return lb.value, ub.value

    # ---- diagnostics.f90, sgm/subgrid_3d.f90 ------------------------------------
    def horizontal_means(self, u, v, w, th, q=None):
        """Returns ubar, vbar, wbar, thbar (kp+2 each) and qbar (nq, kp+2)."""
        K2 = self.grid.kp + 2
        bars = [np.zeros(K2) for _ in range(4)]
        nq = 0 if q is None else q.shape[0]
        qbar = np.zeros((max(nq, 1), K2))
        self._check(self.lib.dcm_horizontal_means(
            self.h, int(nq > 0), nq, self.F(u), self.F(v), self.F(w), self.F(th),
            None if q is None else q.ctypes.data_as(_dp), *[_ptr(b) for b in bars],
            _ptr(qbar)))
        return (*bars, qbar[:nq])

    def divergence_calc(self, u, v, w, div):
        self._check(self.lib.dcm_divergence_calc(self.h, self.F(u), self.F(v), self.F(w),
                                                 self.F(div)))

    def advance_scalar_fields_3d(self, dt, th, sth, q=None, sq=None):
        nq = 0 if q is None else q.shape[0]
        self._check(self.lib.dcm_advance_scalar_fields_3d(
            self.h, float(dt), None if q is None else q.ctypes.data_as(_dp),
            None if sq is None else sq.ctypes.data_as(_dp), self.F(th), self.F(sth), nq,
            int(nq > 0)))

    # ---- mpi_module.f90 ---------------------------------------------------------
    def exchange_full(self, a, lbc, ubc):
        self._check(self.lib.dcm_exchange_full(self.h, self.F(a), float(lbc), float(ubc)))

    def exchange_along_dim(self, a, lbc, ubc):
        self._check(self.lib.dcm_exchange_along_dim(self.h, self.F(a), float(lbc), float(ubc)))

    def exchange_along_dim_wo(self, a):
        self._check(self.lib.dcm_exchange_along_dim_wo(self.h, self.F(a)))

    def exchange_full_wo(self, a):
        self._check(self.lib.dcm_exchange_full_wo(self.h, self.F(a)))

    # ---- sgm/subgrid_3d.f90 -------------------------------------------------------
    def calculate_subgrid_3d(self, lamsq, z0, z0th, u, v, w, zu, zv, zw, th, vism, vist,
                             strain, tau11, tau22, tau33, tau12, tau13, tau23, su, sv, sw, sth,
                             q=None, viss=None, sq=None):
        """calculate_subgrid_3d (sgm/subgrid_3d.f90:38-357): the inout arrays
        are updated in place as the reference does.  q, viss, sq are stacks
        of nq Fortran fields (q[n] is field n); moisture is on when q is
        given.  z(1) is the grid's z[1]."""
        lam = np.ascontiguousarray(lamsq, dtype=np.float64)
        nq = 0 if q is None else q.shape[0]
        self._check(self.lib.dcm_calculate_subgrid_3d(
            self.h, _ptr(lam), float(z0), float(z0th),
            *[self.F(a) for a in (u, v, w, zu, zv, zw, th)], nq,
            None if q is None else q.ctypes.data_as(_dp), self.F(vism), self.F(vist),
            None if viss is None else viss.ctypes.data_as(_dp), self.F(strain),
            *[self.F(a) for a in (tau11, tau22, tau33, tau12, tau13, tau23, su, sv, sw, sth)],
            None if sq is None else sq.ctypes.data_as(_dp), int(nq > 0)))

    # ---- the device-resident time loop (model_driver) ---------------------------
    def upload_state(self, state, dt, ptol=1e-10, kord=3, monotone=True, advection_scheme=1,
                     limiter=0, itmax=9999, nq=0, c_s=(), c_e=(), thbase=0.0, thtop=0.0,
                     forcing=None, precision=0, inner_tol=0.1, viscous=None, precond=0,
                     precond_lo=0.05):
        """viscous = dict(lamsq=(kp+2,), z0=..., z0th=...) switches the
        subgrid model on in sources (dynamics.f90:878-893).  precond = 1
        gives the mixed form's FP32 iterations Chebyshev-weighted Jacobi
        sweeps on [precond_lo, 2] (0: the reference's sweeps)."""
        K2 = self.grid.kp + 2
        cfg = _Config()
        cfg.dt, cfg.ptol = float(dt), float(ptol)
        cfg.advection_scheme, cfg.kord, cfg.monotone = int(advection_scheme), int(kord), \
            int(bool(monotone))
        cfg.limiter, cfg.itmax = int(limiter), int(itmax)
        cfg.moisture, cfg.nq, cfg.ncat = int(nq > 0), int(nq), len(c_s)
        self._cs = (C.c_int * max(1, len(c_s)))(*c_s)
        self._ce = (C.c_int * max(1, len(c_e)))(*c_e)
        cfg.c_s, cfg.c_e = self._cs, self._ce
        cfg.thbase, cfg.thtop, cfg.precision = float(thbase), float(thtop), int(precision)
        cfg.inner_tol = float(inner_tol)
        cfg.precond, cfg.precond_lo = int(precond), float(precond_lo)
        fs, fkeep = self._forcing(forcing)
        if fs is not None:
            cfg.forcing = fs
        if viscous:
            lam = np.ascontiguousarray(viscous["lamsq"], dtype=np.float64)
            cfg.viscous, cfg.lamsq = 1, _ptr(lam)
            cfg.z0, cfg.z0th = float(viscous["z0"]), float(viscous["z0th"])
            fkeep = dict(fkeep or {}, lamsq=lam)
        self._fkeep = fkeep
        sh = self.shape
        f = _Fields()
        for n in ("u", "v", "w", "zu", "zv", "zw", "tu", "tv", "tw", "th", "p"):
            setattr(f, n, self.F(getattr(state, n)))
        # su, sv, sw, sth, psrc and div are recomputed by the first step
        # (sources, the Poisson rhs, the divergence); left NULL they start at
        # zero on the device and nothing crosses PCIe for them
        keep = []
        if nq:
            qs = fortran_stack(state.q)
            sq = fortran_stack([np.zeros(sh, order="F") for _ in range(nq)])
            f.q, f.sq = qs.ctypes.data_as(_dp), sq.ctypes.data_as(_dp)
            keep += [qs, sq]
        self._check(self.lib.dcm_state_upload(self.h, C.byref(cfg), C.byref(f)))
        self._state_keep = keep
        self._nq = nq

    def driver_start(self):
        self._check(self.lib.dcm_driver_start(self.h))

    def last_iters(self):
        """Solver iterations of the last step taken (by step or by an
        Ensemble): dcm_step with zero steps reports the last values."""
        return self.step(0).iters_last

    def step(self, nsteps=1):
        stats = StepStats()
        self._check(self.lib.dcm_step(self.h, int(nsteps), C.byref(stats)))
        return stats

    def solver_graphs(self, on=True):
        """Graph-driven pressure solves (True or 1, the default), the same graphs
        without programmatic dependent launch (2), or the host-polled loop
        (False or 0)."""
        mode = on if isinstance(on, int) and not isinstance(on, bool) else int(bool(on))
        self._check(self.lib.dcm_solver_graphs(self.h, mode))

    def set_small_solver(self, max_points=8192):
        """FP64 solves of domains with at most max_points interior points on
        one thread-block cluster (0: never)."""
        self._check(self.lib.dcm_set_small_solver(self.h, int(max_points)))

    def set_mpdata_shape(self, fuse=False, max_rows=32):
        """MPDATA iterations as one kernel per stage (default) or one fused
        kernel each; max_rows caps the fused kernel's rows per block."""
        self._check(self.lib.dcm_set_mpdata_shape(self.h, int(bool(fuse)), int(max_rows)))

    def solver_limits(self, max_rounds=0, tiny=-1.0):
        """Failure-path limits of later solves: a round budget of the
        graph-driven loop (0: the default, which a solve that behaves never
        reaches; past it DCM_E_TIMEOUT) and the FP64 breakdown threshold of
        |omega| (negative: the reference's tiny, dynamics.f90:321, 414-417)."""
        self._check(self.lib.dcm_solver_limits(self.h, int(max_rounds), float(tiny)))

    def solver_graph_info(self):
        """Whether the graph-driven solves launch their iteration kernels with
        programmatic dependent launch."""
        v = C.c_int(0)
        self._check(self.lib.dcm_solver_graph_info(self.h, C.byref(v)))
        return dict(programmatic_launch=bool(v.value))

    def profile(self, on=True):
        """Enable (and reset) or disable per-kernel-class event timing."""
        self._check(self.lib.dcm_profile_enable(self.h, int(bool(on))))

    def profile_read(self):
        n = len(PROF_CLASSES)
        ms = (C.c_double * n)()
        cnt = (C.c_longlong * n)()
        self._check(self.lib.dcm_profile_read(self.h, ms, cnt, n))
        return {k: (ms[i], cnt[i]) for i, k in enumerate(PROF_CLASSES)}

    def download_state(self, out=None):
        """Returns a dict of host arrays in the current roles.  `out` may hold
        preallocated destinations (e.g. in pinned memory) for any of the
        fields; the others are allocated here."""
        sh = self.shape
        K2 = self.grid.kp + 2
        given = dict(out or {})
        out = {}
        for n in ("u", "v", "w", "zu", "zv", "zw", "tu", "tv", "tw", "th", "p", "su", "sv", "sw",
                  "psrc", "div", "sth"):
            out[n] = given[n] if n in given else np.zeros(sh, order="F")
        bars = {n: (given[n] if n in given else np.zeros(K2))
                for n in ("ubar", "vbar", "wbar", "thbar")}
        f = _Fields()
        for n, a in out.items():
            setattr(f, n, self.F(a))
        for n, a in bars.items():
            setattr(f, n, _ptr(a))
        if self._nq:
            q = fortran_stack([np.zeros(sh, order="F") for _ in range(self._nq)])
            f.q = q.ctypes.data_as(_dp)
            out["q"] = q
        self._check(self.lib.dcm_state_download(self.h, C.byref(f)))
        out.update(bars)
        return out


def _stacked(psi):
    n = psi[0].size
    return all(psi[q].ctypes.data == psi.ctypes.data + q * n * 8 for q in range(psi.shape[0]))


def fortran_stack(fields):
    """Stack nq Fortran-ordered fields into consecutive blocks, the memory
    layout of a Fortran psi(:,:,:,1:nq)."""
    nq = len(fields)
    sh = fields[0].shape
    buf = np.empty((nq,) + sh[::-1], dtype=np.float64)  # C order of the reversed shape
    out = buf.transpose(0, 3, 2, 1)  # each [q] is Fortran ordered with shape sh
    for q, a in enumerate(fields):
        out[q][...] = a
    return out


class Output:
    """The reference's output routine (driver_code.f90:725-1145) for a
    DynamicalCore's resident state: a netCDF classic file written by
    dcm_output_*.  write(time) appends one record of the current state and
    returns at once; the record reaches the file while later steps run.
    x, y, z are the grid coordinates with their halo (default: the grid's),
    trefn the reference temperature profile (kp+2, default zeros), q_names
    the nq tracer names (default q1, q2, ...)."""

    def __init__(self, core, path, x=None, y=None, z=None, trefn=None, q_names=None, nprec=1):
        self.lib = core.lib
        g = core.grid
        nq = getattr(core, "_nq", 0) or 0
        keep = [np.ascontiguousarray(a if a is not None else b, dtype=np.float64)
                for a, b in ((x, g.x), (y, g.y), (z, g.z))]
        tref = None if trefn is None else np.ascontiguousarray(trefn, dtype=np.float64)
        names = b""
        if nq:
            q_names = q_names or ["q%d" % (m + 1) for m in range(nq)]
            names = b"".join(n.encode()[:20].ljust(20) for n in q_names)
        self._keep = (keep, tref, names)
        o = C.c_void_p()
        st = self.lib.dcm_output_open(core.h, os.fsencode(path), *[_ptr(a) for a in keep],
                                      _ptr(tref) if tref is not None else None, int(nq),
                                      names if nq else None, int(nprec), C.byref(o))
        if st:
            raise DCMError(st, self.lib.dcm_status_string(st).decode())
        self.o = o

    def _check(self, st):
        if st:
            msg = self.lib.dcm_output_last_error(self.o)
            raise DCMError(st, (msg or b"").decode() or
                           self.lib.dcm_status_string(st).decode())

    def write(self, time):
        self._check(self.lib.dcm_output_write(self.o, float(time)))

    def flush(self):
        self._check(self.lib.dcm_output_flush(self.o))

    def close(self):
        if getattr(self, "o", None):
            st = self.lib.dcm_output_close(self.o)
            self.o = None
            if st:
                raise DCMError(st, self.lib.dcm_status_string(st).decode())

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Ensemble:
    """Independent domains on one device advanced together, one CUDA graph
    launch per time step (dcm_ensemble_*).  `members[m]` is a DynamicalCore
    view of member m's handle: upload_state / driver_start / download_state /
    tune / step (alone) work on it as on a standalone core."""

    def __init__(self, grids, device=0):
        self.lib = library()
        keeps, structs = zip(*[_grid_struct(g) for g in grids])
        self._keep = keeps
        arr = (_Grid * len(grids))(*structs)
        e = C.c_void_p()
        st = self.lib.dcm_ensemble_create(len(grids), C.cast(arr, C.c_void_p), device, C.byref(e))
        if st:
            raise DCMError(st, self.lib.dcm_status_string(st).decode())
        self.e = e
        self.members = []
        for m, g in enumerate(grids):
            h = C.c_void_p()
            self._check(self.lib.dcm_ensemble_member(self.e, m, C.byref(h)))
            self.members.append(DynamicalCore(g, device, _handle=h))

    def _check(self, st):
        if st:
            msg = self.lib.dcm_ensemble_last_error(self.e)
            raise DCMError(st, (msg or b"").decode() or
                           self.lib.dcm_status_string(st).decode())

    def step(self, nsteps=1):
        stats = EnsembleStats()
        self._check(self.lib.dcm_ensemble_step(self.e, int(nsteps), C.byref(stats)))
        return stats

    def close(self):
        if getattr(self, "e", None):
            for m in self.members:
                m.h = None
            self.lib.dcm_ensemble_destroy(self.e)
            self.e = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
