"""numpy restatement of model_driver's dry time step on one rank
(driver_code.f90:280-295 and 304-676), chaining the numpy restatements of its
routines; an independent check of the oracle's step.

Per step n (advection_scheme = 1; radiation, land surface, the forcings
and the microphysics off; passive q categories and the subgrid model
optional):
  sth = 0; horizontal_means; divergence_calc; sources;
  exchange_along_dim_wo(psrc); bicgstab(p, psrc); exchange_along_dim_wo(p);
  adv_ref_state(th) + exchange_full(th, 0, 0); mpdata_3d(th, t1, t2);
  mpdata_vec_3d of each q category (with sq = 0);
  advance_momentum(2 dt, tu, tv, tw); advance_scalar_fields_3d(th, q);
  the 0.99 / 0.01 filter of u and zu; the rotation of the u, zu, tu roles by
  n mod 3; exchange_full(u, v, w, 0, 0) and the velocity rows.
horizontal_means forms every level's mean (the reference's Allreduce count
leaves the top levels of its last mean unreduced; with the reference's
nq >= 1 that is a q mean, which the dry step does not use).
"""
import numpy as np

import bicgstab_np
import dynamics_np
import mpdata_np
from helpers import cases


def exchange_along_dim_wo(a):
    """Single rank: the x and y faces of levels 1..kp take their periodic
    images (mpi_module.f90:1441-1456); the top and bottom planes stay."""
    kp, jp, ip = a.shape[0] - 2, a.shape[1] - 2, a.shape[2] - 2
    a[1:kp + 1, 1:jp + 1, 0] = a[1:kp + 1, 1:jp + 1, ip]
    a[1:kp + 1, 1:jp + 1, ip + 1] = a[1:kp + 1, 1:jp + 1, 1]
    a[1:kp + 1, 0, 1:ip + 1] = a[1:kp + 1, jp, 1:ip + 1]
    a[1:kp + 1, jp + 1, 1:ip + 1] = a[1:kp + 1, 1, 1:ip + 1]


def horizontal_means(a):
    """per-level mean over the interior columns: the level's sum in array
    element order (diagnostics.f90:64-70), divided by ip*jp (:83-88)"""
    jp, ip = a.shape[1] - 2, a.shape[2] - 2
    out = np.empty(a.shape[0])
    for k in range(a.shape[0]):
        out[k] = np.cumsum(a[k, 1:jp + 1, 1:ip + 1].ravel(order="F"))[-1] / float(ip * jp)
    return out


class Driver:
    def __init__(self, g, state, dt, ptol=1e-10, kord=3, monotone=True, c_s=(), c_e=(),
                 viscous=None):
        self.g, self.dt, self.ptol, self.kord, self.monotone = g, dt, ptol, kord, monotone
        # viscous = dict(lamsq, z0, z0th): the subgrid model inside sources, with
        # vism, vist and strain kept between steps
        self.viscous = None
        if viscous:
            self.viscous = dict(viscous, **{n: np.zeros(g.shape, order="F")
                                           for n in ("vism", "vist", "strain")})
        self.cats = list(zip(c_s, c_e))
        self.q = [np.asfortranarray(a).copy(order="F") for a in state.q] if c_s else []
        self.q1, self.q2 = np.zeros(len(self.q)), np.zeros(len(self.q))
        sh = g.shape
        self.buf = {n: np.asfortranarray(getattr(state, n)).copy(order="F")
                    for n in ("u", "v", "w", "zu", "zv", "zw", "tu", "tv", "tw")}
        self.th = np.asfortranarray(state.th).copy(order="F")
        self.p = np.asfortranarray(state.p).copy(order="F")
        for n in ("su", "sv", "sw", "psrc", "div", "sth"):
            setattr(self, n, np.zeros(sh, order="F"))
        self.t1 = self.t2 = 0.0
        self.n = 0
        # the roles of driver_code.f90:280-282
        self.role = {c: {"": self.buf[c], "z": self.buf["z" + c], "t": self.buf["t" + c]}
                     for c in ("u", "v", "w")}
        self.fixed = {c: (self.buf[c], self.buf["z" + c], self.buf["t" + c])
                      for c in ("u", "v", "w")}

    def start(self):
        """the rows of driver_code.f90:285-295"""
        kp = self.g.kp
        zu, zv, zw = (self.role[c]["z"] for c in ("u", "v", "w"))
        zw[0] = -zw[1]
        zu[1] = 0.0
        zv[1] = 0.0
        zw[kp] = -zw[kp - 1]
        zw[kp + 1] = 0.0
        zu[kp] = 0.0
        zv[kp] = 0.0

    def step(self):
        g, dt = self.g, self.dt
        kp = g.kp
        self.n += 1
        n = self.n
        u, v, w = (self.role[c][""] for c in ("u", "v", "w"))
        zu, zv, zw = (self.role[c]["z"] for c in ("u", "v", "w"))
        tu, tv, tw = (self.role[c]["t"] for c in ("u", "v", "w"))
        self.sth[...] = 0.0
        self.bars = [horizontal_means(a) for a in (u, v, w, self.th)]
        dynamics_np.divergence_calc(g, u, v, w, self.div)
        dynamics_np.sources(g, *self.bars, zu, zv, zw, u, v, w, self.th, self.su, self.sv,
                            self.sw, self.sth, self.psrc, viscous=self.viscous)
        exchange_along_dim_wo(self.psrc)
        st, self.iters, self.err = bicgstab_np.bicgstab(g, self.p, self.psrc, self.sw,
                                                        self.ptol)
        assert st == 0
        exchange_along_dim_wo(self.p)
        dynamics_np.adv_ref_state(g, dt, w, self.th, g.thetan)
        cases.exchange_full(self.th, 0.0, 0.0)
        self.t1, self.t2 = mpdata_np.mpdata_3d(g, dt, u, v, w, self.th, self.t1, self.t2,
                                               self.kord, self.monotone, 0)
        for cs, ce in self.cats:  # driver_code.f90:577-597
            mpdata_np.mpdata_vec_3d(g, dt, u, v, w, self.q[cs - 1:ce], self.q1[cs - 1:ce],
                                    self.q2[cs - 1:ce], self.kord, self.monotone, 0)
        dynamics_np.advance_momentum(g, 2.0 * dt, tu, tv, tw, zu, zv, zw, self.su, self.sv,
                                     self.sw, self.p)
        self.th[...] = self.th + self.sth * dt
        for a in self.q:  # sq = 0: the driver zeroes it and nothing adds to it here
            a[...] = a + 0.0 * dt
        for a, za in ((u, zu), (v, zv), (w, zw)):
            tmp = 0.99 * a + 0.01 * za
            za[...] = 0.01 * a + 0.99 * za
            a[...] = tmp
        for c in ("u", "v", "w"):
            cur, prev, nxt = self.fixed[c]
            if n % 3 == 1:
                self.role[c] = {"": nxt, "z": cur, "t": prev}
            elif n % 3 == 2:
                self.role[c] = {"": prev, "z": nxt, "t": cur}
            else:
                self.role[c] = {"": cur, "z": prev, "t": nxt}
        u, v, w = (self.role[c][""] for c in ("u", "v", "w"))
        for a in (u, v, w):
            cases.exchange_full(a, 0.0, 0.0)
        w[0] = 0.0
        u[0] = -u[1]
        v[0] = -v[1]
        w[kp + 1] = 0.0
        u[kp + 1] = u[kp]
        v[kp + 1] = v[kp]

    def fields(self):
        out = {}
        for c in ("u", "v", "w"):
            out[c] = self.role[c][""]
            out["z" + c] = self.role[c]["z"]
            out["t" + c] = self.role[c]["t"]
        for n in ("th", "p", "su", "sv", "sw", "psrc", "div", "sth"):
            out[n] = getattr(self, n)
        for n, a in zip(("ubar", "vbar", "wbar", "thbar"), self.bars):
            out[n] = a
        if self.q:
            out["q"] = self.q
        if self.viscous:
            for n in ("vism", "vist", "strain"):
                out[n] = self.viscous[n]
        return out
