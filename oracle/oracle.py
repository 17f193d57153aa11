"""ctypes binding of the CPU restatement (dcm_oracle.c).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
CPU-baseline / reference legs of bench.py, as the parity reference.  PARITY UNPINNED
(no Fortran compiler in this image; the reference ships no golden vectors).

The methods mirror the product binding (dynamical-cloud-model_b200) name for
name so a test can run the same call on both and compare.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libdcm_oracle.so")
_dp = C.POINTER(C.c_double)


def build(force=False):
    src = [os.path.join(HERE, f)
           for f in ("dcm_oracle.c", "dcm_oracle_sgm.c", "dcm_oracle_col.c", "dcm_oracle.h",
                     "Makefile")]
    if force or not os.path.exists(LIBPATH) or \
            any(os.path.getmtime(s) > os.path.getmtime(LIBPATH) for s in src):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIBPATH


class _OGrid(C.Structure):
    _fields_ = [("ip", C.c_int), ("jp", C.c_int), ("kp", C.c_int)] + [
        (n, _dp) for n in ("dx", "dxn", "dy", "dyn", "dz", "dzn", "rhoa", "rhoan", "theta",
                           "thetan", "xg", "yg", "zg")]


class _OForcing(C.Structure):
    _fields_ = [("damping_layer", C.c_int), ("forcing", C.c_int), ("divergence", C.c_int),
                ("dampfacn", _dp), ("dampfac", _dp), ("u_force", _dp), ("v_force", _dp),
                ("w_subs", _dp), ("forcing_tau", C.c_double)]


class _OViscous(C.Structure):
    _fields_ = [("viscous", C.c_int), ("lamsq", _dp), ("z0", C.c_double), ("z0th", C.c_double)]


class _OConfig(C.Structure):
    _fields_ = [("dt", C.c_double), ("ptol", C.c_double), ("advection_scheme", C.c_int),
                ("kord", C.c_int), ("monotone", C.c_int), ("limiter_variant", C.c_int),
                ("moisture", C.c_int), ("nq", C.c_int), ("ncat", C.c_int),
                ("c_s", C.POINTER(C.c_int)), ("c_e", C.POINTER(C.c_int)),
                ("thbase", C.c_double), ("thtop", C.c_double), ("forcing", _OForcing),
                ("viscous", _OViscous)]


class _OState(C.Structure):
    _fields_ = [(n, _dp) for n in ("ut", "vt", "wt", "zut", "zvt", "zwt", "tut", "tvt", "twt",
                                   "th", "p", "su", "sv", "sw", "psrc", "div", "sth", "q", "sq",
                                   "ubar", "vbar", "wbar", "thbar", "qbar")] + [
        ("t1", C.c_double), ("t2", C.c_double), ("q1", _dp), ("q2", _dp), ("n", C.c_int),
        ("bicgstab_first", C.c_int), ("last_iters", C.c_int), ("last_err", C.c_double),
        ("vism", _dp), ("vist", _dp), ("strain", _dp)]


_lib = None


def library():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(LIBPATH)
        L = _lib
        L.orc_bicgstab.restype = C.c_int
        L.orc_model_step.restype = C.c_int
        L.orc_inn_prod.restype = C.c_double
        L.orc_set_threads.argtypes = [C.c_int, C.c_int]
        L.orc_set_breakdown_tiny.argtypes = [C.c_double]
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _F(a):
    assert a.dtype == np.float64 and a.flags.f_contiguous, "Fortran float64 field expected"
    return a.ctypes.data_as(_dp)


def set_threads(n, parallel_reductions=False):
    library().orc_set_threads(int(n), int(bool(parallel_reductions)))


def set_breakdown_tiny(tiny=-1.0):
    """Breakdown threshold of |omega| in later bicgstab calls (negative: the
    reference's 1.e-16, dynamics.f90:321)."""
    library().orc_set_breakdown_tiny(float(tiny))


class OracleCore:
    def __init__(self, grid):
        self.lib = library()
        self.grid = grid
        self.shape = (grid.kp + 2, grid.jp + 2, grid.ip + 2)
        self._keep = [np.ascontiguousarray(getattr(grid, n), dtype=np.float64)
                      for n in ("dx", "dxn", "dy", "dyn", "dz", "dzn", "rhoa", "rhoan", "theta",
                                "thetan", "x", "y", "z")]
        self.g = _OGrid(grid.ip, grid.jp, grid.kp, *[a.ctypes.data_as(_dp) for a in self._keep])
        self.first_call = C.c_int(1)

    def _forcing(self, f):
        if not f:
            return None, None
        keep = {}
        fs = _OForcing()
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

    # dynamics.f90
    def bicgstab(self, x, b, sw, tol, test_solver=False, itmax=9999):
        it = C.c_int(0)
        err = C.c_double(0.0)
        st = self.lib.orc_bicgstab(C.byref(self.g), _F(x), _F(b), _F(sw), C.c_double(tol),
                                   int(bool(test_solver)), C.byref(self.first_call), int(itmax),
                                   C.byref(it), C.byref(err))
        return st, it.value, err.value

    def mat_ax(self, x, ax):
        self.lib.orc_mat_ax(C.byref(self.g), _F(x), _F(ax))

    def sources(self, ubar, vbar, wbar, thbar, zu, zv, zw, u, v, w, th, su, sv, sw, sth, rhs,
                forcing=None):
        fs, keep = self._forcing(forcing)
        z = np.zeros(self.shape, order="F")
        self.lib.orc_sources(C.byref(self.g), C.byref(fs) if fs is not None else None,
                             _p(ubar), _p(vbar), _p(wbar), _p(thbar),
                             *[_F(a if a is not None else z) for a in (zu, zv, zw)],
                             _F(u), _F(v), _F(w), _F(th), _F(su), _F(sv), _F(sw), _F(sth),
                             _F(rhs))

    def sources_viscous(self, ubar, vbar, wbar, thbar, zu, zv, zw, u, v, w, th, su, sv, sw,
                        sth, rhs, lamsq, z0, z0th, vism, vist, strain, q=None, sq=None,
                        forcing=None):
        """sources with viscous = .true.: the subgrid model in place of the
        full exchange of su, sv, sw, sth (dynamics.f90:878-893)."""
        fs, keep = self._forcing(forcing)
        vis = _OViscous(1, None, float(z0), float(z0th))
        lam = np.ascontiguousarray(lamsq, dtype=np.float64)
        vis.lamsq = lam.ctypes.data_as(_dp)
        nq = 0 if q is None else q.shape[0]
        self.lib.orc_sources_viscous(
            C.byref(self.g), C.byref(fs) if fs is not None else None, C.byref(vis),
            _p(ubar), _p(vbar), _p(wbar), _p(thbar), _F(zu), _F(zv), _F(zw), _F(u), _F(v),
            _F(w), _F(th), nq, None if q is None else q.ctypes.data_as(_dp), int(nq > 0),
            _F(vism), _F(vist), _F(strain), _F(su), _F(sv), _F(sw), _F(sth),
            None if sq is None else sq.ctypes.data_as(_dp), _F(rhs))

    # sgm/subgrid_3d.f90
    def calculate_subgrid_3d(self, lamsq, z0, z0th, u, v, w, zu, zv, zw, th, vism, vist,
                             strain, tau11, tau22, tau33, tau12, tau13, tau23, su, sv, sw, sth,
                             q=None, viss=None, sq=None):
        """calculate_subgrid_3d (sgm/subgrid_3d.f90:38-357); z is the grid's z.
        q, viss, sq: stacks of nq Fortran fields (moisture on when q is given)."""
        lam = np.ascontiguousarray(lamsq, dtype=np.float64)
        nq = 0 if q is None else q.shape[0]
        self.lib.orc_calculate_subgrid_3d(
            C.byref(self.g), _p(lam), C.c_double(z0), C.c_double(z0th),
            *[_F(a) for a in (u, v, w, zu, zv, zw, th)], nq,
            None if q is None else q.ctypes.data_as(_dp), _F(vism), _F(vist),
            None if viss is None else viss.ctypes.data_as(_dp), _F(strain),
            *[_F(a) for a in (tau11, tau22, tau33, tau12, tau13, tau23, su, sv, sw, sth)],
            None if sq is None else sq.ctypes.data_as(_dp), int(nq > 0))

    def exchange_full_wo(self, a):
        self.lib.orc_exchange_full_wo(C.byref(self.g), _F(a))

    def advance_momentum(self, dt, u, v, w, zu, zv, zw, su, sv, sw, p):
        self.lib.orc_advance_momentum(C.byref(self.g), C.c_double(dt),
                                      *[_F(a) for a in (u, v, w, zu, zv, zw, su, sv, sw, p)])

    # advection
    def first_order_upstream_3d(self, dt, u, v, w, psi, neumann=0):
        self.lib.orc_first_order_upstream_3d(C.byref(self.g), C.c_double(dt), _F(u), _F(v),
                                             _F(w), _F(psi), int(neumann))

    def mpdata_3d(self, dt, u, v, w, psi, lbc, ubc, kord, monotone, neumann=0, limiter=0):
        lb, ub = C.c_double(lbc), C.c_double(ubc)
        self.lib.orc_mpdata_3d(C.byref(self.g), C.c_double(dt), _F(u), _F(v), _F(w), _F(psi),
                               C.byref(lb), C.byref(ub), int(kord), int(bool(monotone)),
                               int(neumann), int(limiter))
        return lb.value, ub.value

    def mpdata_vec_3d(self, dt, u, v, w, psi, lbc, ubc, kord, monotone, neumann=0, limiter=0):
        self.lib.orc_mpdata_vec_3d(C.byref(self.g), C.c_double(dt), _F(u), _F(v), _F(w),
                                   psi.ctypes.data_as(_dp), psi.shape[0], _p(lbc), _p(ubc),
                                   int(kord), int(bool(monotone)), int(neumann), int(limiter))

    def adv_ref_state(self, dt, w, psi, psi_ref):
        ref = np.ascontiguousarray(psi_ref, dtype=np.float64)
        self.lib.orc_adv_ref_state(C.byref(self.g), C.c_double(dt), _F(w), _F(psi), _p(ref))

    def mpdata_3d_add(self, dt, u, v, w, psi, psi_1d, lbc, ubc, kord, monotone, neumann=0,
                      limiter=0):
        lb, ub = C.c_double(lbc), C.c_double(ubc)
        prof = np.ascontiguousarray(psi_1d, dtype=np.float64)
        self.lib.orc_mpdata_3d_add(C.byref(self.g), C.c_double(dt), _F(u), _F(v), _F(w),
                                   _F(psi), _p(prof), C.byref(lb), C.byref(ub), int(kord),
                                   int(bool(monotone)), int(neumann), int(limiter))
        return lb.value, ub.value

    # diagnostics
    def horizontal_means(self, u, v, w, th, q=None):
        K2 = self.grid.kp + 2
        bars = [np.zeros(K2) for _ in range(4)]
        nq = 0 if q is None else q.shape[0]
        qbar = np.zeros((max(nq, 1), K2))
        self.lib.orc_horizontal_means(C.byref(self.g), int(nq > 0), nq, _F(u), _F(v), _F(w),
                                      _F(th), None if q is None else q.ctypes.data_as(_dp),
                                      *[_p(b) for b in bars], _p(qbar))
        return (*bars, qbar[:nq])

    def divergence_calc(self, u, v, w, div):
        self.lib.orc_divergence_calc(C.byref(self.g), _F(u), _F(v), _F(w), _F(div))

    def advance_scalar_fields_3d(self, dt, th, sth, q=None, sq=None):
        nq = 0 if q is None else q.shape[0]
        self.lib.orc_advance_scalar_fields_3d(
            C.byref(self.g), C.c_double(dt), None if q is None else q.ctypes.data_as(_dp),
            None if sq is None else sq.ctypes.data_as(_dp), _F(th), _F(sth), nq, int(nq > 0))

    def exchange_full(self, a, lbc, ubc):
        self.lib.orc_exchange_full(C.byref(self.g), _F(a), C.c_double(lbc), C.c_double(ubc))

    def exchange_along_dim(self, a, lbc, ubc):
        self.lib.orc_exchange_along_dim(C.byref(self.g), _F(a), C.c_double(lbc),
                                        C.c_double(ubc))

    def exchange_along_dim_wo(self, a):
        self.lib.orc_exchange_along_dim_wo(C.byref(self.g), _F(a))


class OracleModel:
    """model_driver's time loop on the CPU restatement."""

    def __init__(self, grid, state, dt, ptol=1e-10, kord=3, monotone=True, advection_scheme=1,
                 limiter=0, nq=0, c_s=(), c_e=(), thbase=0.0, thtop=0.0, forcing=None,
                 viscous=None):
        self.lib = library()
        self.core = OracleCore(grid)
        sh = self.core.shape
        K2 = grid.kp + 2
        self.f = {n: np.asfortranarray(getattr(state, n)).copy(order="F")
                  for n in ("u", "v", "w", "zu", "zv", "zw", "tu", "tv", "tw", "th", "p")}
        for n in ("su", "sv", "sw", "psrc", "div", "sth"):
            self.f[n] = np.zeros(sh, order="F")
        self.bars = {n: np.zeros(K2) for n in ("ubar", "vbar", "wbar", "thbar")}
        self.nq = nq
        if nq:
            from_stack = _fortran_stack
            self.q = from_stack(state.q)
            self.sq = from_stack([np.zeros(sh, order="F") for _ in range(nq)])
            self.qbar = np.zeros(nq * K2)
            self.q1 = np.zeros(nq)
            self.q2 = np.zeros(nq)
        s = _OState()
        roles = dict(ut="u", vt="v", wt="w", zut="zu", zvt="zv", zwt="zw", tut="tu", tvt="tv",
                     twt="tw")
        for cn, pn in roles.items():
            setattr(s, cn, _F(self.f[pn]))
        for n in ("th", "p", "su", "sv", "sw", "psrc", "div", "sth"):
            setattr(s, n, _F(self.f[n]))
        for n, a in self.bars.items():
            setattr(s, n, _p(a))
        if nq:
            s.q, s.sq = self.q.ctypes.data_as(_dp), self.sq.ctypes.data_as(_dp)
            s.qbar, s.q1, s.q2 = _p(self.qbar), _p(self.q1), _p(self.q2)
        s.t1 = s.t2 = 0.0
        s.n = 0
        s.bicgstab_first = 1
        self.s = s
        cfg = _OConfig()
        cfg.dt, cfg.ptol = dt, ptol
        cfg.advection_scheme, cfg.kord, cfg.monotone = advection_scheme, kord, int(bool(monotone))
        cfg.limiter_variant = limiter
        cfg.moisture, cfg.nq, cfg.ncat = int(nq > 0), nq, len(c_s)
        self._cs = (C.c_int * max(1, len(c_s)))(*c_s)
        self._ce = (C.c_int * max(1, len(c_e)))(*c_e)
        cfg.c_s, cfg.c_e = self._cs, self._ce
        cfg.thbase, cfg.thtop = thbase, thtop
        fs, self._fkeep = self.core._forcing(forcing)
        if fs is not None:
            cfg.forcing = fs
        if viscous:
            # viscous = dict(lamsq=(kp+2,), z0=..., z0th=...): the subgrid model
            self._lamsq = np.ascontiguousarray(viscous["lamsq"], dtype=np.float64)
            cfg.viscous = _OViscous(1, self._lamsq.ctypes.data_as(_dp),
                                    float(viscous["z0"]), float(viscous["z0th"]))
            for n in ("vism", "vist", "strain"):
                self.f[n] = np.zeros(sh, order="F")
                setattr(s, n, _F(self.f[n]))
        self.cfg = cfg

    def driver_start(self):
        self.lib.orc_driver_start(C.byref(self.core.g), C.byref(self.s))

    def step(self, nsteps=1):
        for _ in range(nsteps):
            st = self.lib.orc_model_step(C.byref(self.core.g), C.byref(self.cfg),
                                         C.byref(self.s))
            if st:
                raise RuntimeError("oracle step failed with status %d" % st)
        return self.s.last_iters, self.s.last_err

    def fields(self):
        """Current roles (u, zu, tu ...) after the rotation, plus scalars."""
        m = self.s.n % 3
        order = [("u", "zu", "tu"), ("tu", "u", "zu"), ("zu", "tu", "u")][m]
        out = {}
        for c, names in (("u", ("u", "zu", "tu")), ("v", ("v", "zv", "tv")),
                         ("w", ("w", "zw", "tw"))):
            bufs = {"u": self.f[names[0]], "zu": self.f[names[1]], "tu": self.f[names[2]]}
            out[c] = bufs[order[0]]
            out["z" + c] = bufs[order[1]]
            out["t" + c] = bufs[order[2]]
        for n in ("th", "p", "su", "sv", "sw", "psrc", "div", "sth"):
            out[n] = self.f[n]
        out.update(self.bars)
        if self.nq:
            out["q"] = self.q
        return out


def mpdata_vec_1d_columns(dt, nsub, dz, dzn, rhoa, rhoan, w, psi, kord=1, monotone=False,
                          neumann=0, l_h=1, r_h=1):
    """The PAMM sedimentation transport of ncol columns, in place on psi
    (dcm_oracle_col.c: mpdata_vec_1d, pamm/sfvt/advection_1d.F90:463-778,
    nsub[c] passes of dt[c]/nsub[c]).  w: (ncol, kp+l_h+r_h), each row
    w(-l_h+1:kp+r_h); psi: (ncol, nq, kp+2 r_h), each column's
    psi_in(-r_h+1:kp+r_h, 1:nq); dz, dzn, rhoa, rhoan: (kp+l_h+r_h,) shared
    or (ncol, kp+l_h+r_h) per column."""
    L = library()
    ncol, nq, npsi = psi.shape
    kp = npsi - 2 * r_h
    nw = kp + l_h + r_h
    assert psi.dtype == np.float64 and psi.flags.c_contiguous
    w = np.ascontiguousarray(w, dtype=np.float64)
    assert w.shape == (ncol, nw)
    met = [np.ascontiguousarray(a, dtype=np.float64) for a in (dz, dzn, rhoa, rhoan)]
    stride = nw if met[0].ndim == 2 else 0
    for a in met:
        assert a.shape == ((ncol, nw) if stride else (nw,))
    dt = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, dtype=np.float64), (ncol,)))
    ns = None if nsub is None else np.ascontiguousarray(
        np.broadcast_to(np.asarray(nsub, dtype=np.int32), (ncol,)))
    L.orc_mpdata_vec_1d_columns(
        C.c_int(ncol), C.c_int(kp), C.c_int(nq), C.c_int(l_h), C.c_int(r_h), _p(dt),
        None if ns is None else ns.ctypes.data_as(C.POINTER(C.c_int)), *[_p(a) for a in met],
        C.c_int(stride), _p(w), _p(psi), C.c_int(kord), C.c_int(int(bool(monotone))),
        C.c_int(neumann))
    return psi


def _fortran_stack(fields):
    nq = len(fields)
    sh = fields[0].shape
    buf = np.empty((nq,) + sh[::-1], dtype=np.float64)
    out = buf.transpose(0, 3, 2, 1)
    for q, a in enumerate(fields):
        out[q][...] = a
    return out
