"""Independent numpy restatement of the PAMM sedimentation transport,
mpdata_vec_1d with first_order_upstream_1d (pamm/sfvt/advection_1d.F90:35-74,
463-778), written array statement by array statement from the Fortran, to
pin the C oracle (oracle/dcm_oracle_col.c) bit for bit.

Arrays of one column are indexed from the Fortran lower bound: w[k + l_h - 1]
is w(k); psi[n, k + r_h - 1] is psi_in(k, n+1).
"""
import numpy as np

SMALL = 1e-60  # pamm/sfvt/advection_1d.F90:18


def _upstream(dt, dzn, rhoa, rhoan, kp, w, psi, neumann, ow, op):
    """first_order_upstream_1d (:35-74) on one field; ow, op: index of level
    0 in w-like arrays and in psi."""
    k = np.arange(1, kp + 1)
    a = lambda x, kk: x[kk + ow]  # noqa: E731
    p = lambda kk: psi[kk + op]  # noqa: E731
    wk, wm = a(w, k), a(w, k - 1)
    den = 2.0 * a(dzn, k) * a(rhoan, k)
    fz_r = ((wk + np.abs(wk)) * a(rhoa, k) * p(k) + (wk - np.abs(wk)) * a(rhoa, k) * p(k + 1)) \
        * dt / den
    fz_l = ((wm + np.abs(wm)) * a(rhoa, k - 1) * p(k - 1) +
            (wm - np.abs(wm)) * a(rhoa, k - 1) * p(k)) * dt / den
    if neumann == 1:
        fz_l[0] = fz_r[0]
        fz_r[kp - 1] = fz_l[kp - 1]
    elif neumann == 2:
        fz_l[0] = -fz_r[0]
        fz_r[kp - 1] = -fz_l[kp - 1]
    psi[1 + op:kp + 1 + op] = psi[1 + op:kp + 1 + op] - (fz_r - fz_l)


def mpdata_vec_1d(dt, dz, dzn, rhoa, rhoan, kp, nq, l_h, r_h, w, psi_in, kord, monotone,
                  neumann):
    """mpdata_vec_1d (:463-778) on one column, in place on psi_in (nq, kp+2 r_h)."""
    ow, op = l_h - 1, r_h - 1
    nw = kp + l_h + r_h
    a = lambda x, kk: x[kk + ow]  # noqa: E731
    minglobal = np.array([np.min(psi_in[n, 1 + op:kp + 1 + op]) for n in range(nq)])
    for n in range(nq):
        psi_in[n, :] = psi_in[n, :] - minglobal[n]
    psi_sum = 0.0
    for v in psi_in[0, 1 + op:kp + 1 + op]:  # the intrinsic sum, in index order
        psi_sum += v
    if psi_sum < SMALL:
        for n in range(nq):
            psi_in[n, :] = psi_in[n, :] + minglobal[n]
        return
    w_store1 = np.zeros(nw)
    w_store2 = np.zeros(nw)
    wt, wt_sav = w, w_store1
    psi = psi_in[0].copy() if kord > 1 else None
    psi_old = psi_in[0]  # a view: follows the field through the passes
    k = np.arange(1, kp + 1)
    it2 = 0
    for it in range(1, kord + 1):
        if it > 1:
            it2 += 1
            g_bar3 = 0.5 * (a(rhoan, k) + a(rhoan, k + 1))
            wk = a(wt, k)
            po1, po0 = psi_old[k + 1 + op], psi_old[k + op]
            v = (np.abs(wk) * a(dz, k) - dt * (a(rhoa, k) / g_bar3) * wk * wk) * (po1 - po0) \
                / (po1 + po0 + SMALL) / a(dzn, k) - 0.0
            v = v - 0.25 * dt * wk * ((a(rhoa, k + 1) * a(wt, k + 1) -
                                       a(rhoa, k - 1) * a(wt, k - 1)) / a(dz, k - 1) + 0.0) \
                / g_bar3
            wt_sav[k + ow] = v
            if it2 % 2 == 1:
                wt, wt_sav = w_store1, w_store2
            else:
                wt, wt_sav = w_store2, w_store1
            wt[0 + ow] = wt[1 + ow]
            wt[kp + ow] = wt[kp - 1 + ow]
            wt[kp + 1 + ow] = wt[kp - 1 + ow]
        if it > 1 and monotone:
            it2 += 1
            cands = [psi[k - 1 + op], psi[k + op], psi[k + 1 + op],
                     psi_old[k - 1 + op], psi_old[k + op], psi_old[k + 1 + op]]
            psi_max = np.maximum.reduce(cands)
            psi_min = np.minimum.reduce(cands)
            wm, wk = a(wt, k - 1), a(wt, k)
            pm, pc, pp = psi_old[k - 1 + op], psi_old[k + op], psi_old[k + 1 + op]
            denom1 = dt * (np.maximum(wm, 0.0) * a(rhoa, k - 1) * pm -
                           np.minimum(wk, 0.0) * a(rhoa, k) * pp) / a(dzn, k) + SMALL
            denom2 = dt * (np.maximum(wk, 0.0) * a(rhoa, k) * pc -
                           np.minimum(wm, 0.0) * a(rhoa, k - 1) * pc) / a(dzn, k) + SMALL
            beta_up = np.zeros(kp + 2)  # levels 0 .. kp+1
            beta_down = np.zeros(kp + 2)
            beta_up[1:kp + 1] = a(rhoan, k) * (psi_max - pc) / denom1
            beta_down[1:kp + 1] = a(rhoan, k) * (pc - psi_min) / denom2
            wt_sav[k + ow] = np.minimum(np.minimum(1.0, beta_down[1:kp + 1]), beta_up[2:kp + 2]) \
                * np.maximum(wk, 0.0) + \
                np.minimum(np.minimum(1.0, beta_up[1:kp + 1]), beta_down[2:kp + 2]) \
                * np.minimum(wk, 0.0)
            wt, wt_sav = w_store2, w_store1
            wt[0 + ow] = wt[1 + ow]
            wt[kp + ow] = wt[kp - 1 + ow]
            wt[kp + 1 + ow] = wt[kp - 1 + ow]
        for n in range(nq):
            _upstream(dt, dzn, rhoa, rhoan, kp, wt, psi_in[n], neumann, ow, op)
            psi_in[n, 0 + op] = 0.0
            psi_in[n, kp + 1 + op] = 0.0
    for n in range(nq):
        psi_in[n, :] = psi_in[n, :] + minglobal[n]


def columns(dt, nsub, dz, dzn, rhoa, rhoan, w, psi, kord=1, monotone=False, neumann=0, l_h=1,
            r_h=1):
    """ncol columns, nsub[c] passes of dt[c]/nsub[c] each, in place on psi."""
    ncol, nq, npsi = psi.shape
    kp = npsi - 2 * r_h
    dt = np.broadcast_to(np.asarray(dt, dtype=np.float64), (ncol,))
    ns = np.ones(ncol, dtype=int) if nsub is None else np.broadcast_to(np.asarray(nsub), (ncol,))
    per = np.ndim(dz) == 2
    for c in range(ncol):
        m = [x[c] if per else x for x in (dz, dzn, rhoa, rhoan)]
        for _ in range(int(ns[c])):
            mpdata_vec_1d(dt[c] / float(ns[c]), *m, kp, nq, l_h, r_h, w[c], psi[c], kord,
                          monotone, neumann)
    return psi
