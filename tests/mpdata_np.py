"""Array-at-a-time numpy restatement of the reference's mpdata_3d
(pamm/sfvt/advection_3d.F90:219-714) and mpdata_vec_3d (:1250-1753) on one
rank, an independent check of the oracle's C restatement:

* the positive-definite shift by the global minimum (:271-285);
* for each pass after the first, the antidiffusive velocities of the
  divergent-flow MPDATA with G = rho (:319-507; Smolarkiewicz 1984, eqs. 13,
  14 and 38), written into the store the rotation of :509-527 selects;
* with monotone, the FCT limiter (:542-675; Smolarkiewicz and Grabowski 1990,
  eqs. 18-20), whose bounds also take the field as it was at entry (the copy
  psi_store);
* the donor-cell pass (first_order_upstream_3d) and exchange_full of the
  field after every pass (:683-700);
* mpdata_vec_3d: the same passes with the velocities and bounds of the
  category's first field, the donor cell and the exchange for every field,
  and a shift per field by the minimum of its interior.

Every expression keeps the reference's parenthesisation and left-to-right
evaluation, so the result is bit for bit the reference's arithmetic in IEEE
double without fused multiply-adds.
"""
import numpy as np

import bicgstab_np
import dynamics_np
from helpers import cases

SMALL = 1e-60  # small, advection_3d.F90:19


def _k(a):
    return a[:, None, None]


def _antidiffusive(g, dt, ut, vt, wt, po, us, vs, ws):
    """us, vs, ws (interior) from ut, vt, wt and psi_old = po, :319-507."""
    kp = g.kp
    K, Km, Kp = slice(1, kp + 1), slice(0, kp), slice(2, kp + 2)
    J, Jm, Jp = slice(1, -1), slice(0, -2), slice(2, None)
    I, Im, Ip = slice(1, -1), slice(0, -2), slice(2, None)
    ra, rn = _k(g.rhoa), _k(g.rhoan)
    ra_k, ra_km, ra_kp = ra[K], ra[Km], ra[Kp]
    rn_k, rn_kp = rn[K], rn[Kp]
    dx_i = g.dx[None, None, I]
    dx_im = g.dx[None, None, Im]
    dy_j = g.dy[None, J, None]
    dy_jm = g.dy[None, Jm, None]
    dz_k, dz_km = _k(g.dz[K]), _k(g.dz[Km])
    dxn_i, dxn_im = g.dxn[None, None, I], g.dxn[None, None, Im]
    dyn_j, dyn_jm = g.dyn[None, J, None], g.dyn[None, Jm, None]
    dzn_k, dzn_km = _k(g.dzn[K]), _k(g.dzn[Km])
    g1 = rn_k
    g2 = rn_k
    g3 = 0.5 * (rn_k + rn_kp)

    def U(k, j, i):
        return ut[k, j, i]

    def V(k, j, i):
        return vt[k, j, i]

    def W(k, j, i):
        return wt[k, j, i]

    def P(k, j, i):
        return po[k, j, i]

    u_div1 = ((ra_k * (W(K, J, I) + W(K, J, Ip)) - ra_km * (W(Km, J, I) + W(Km, J, Ip))) /
              (dz_km * g1) +
              (rn_k * (V(K, J, I) + V(K, J, Ip) - V(K, Jm, I) - V(K, Jm, Ip))) / (dy_jm * g1))
    u_div2 = ((ra_k * (W(K, J, I) + W(K, Jp, I)) - ra_km * (W(Km, J, I) + W(Km, Jp, I))) /
              (dz_km * g2) +
              (rn_k * (U(K, J, I) + U(K, Jp, I) - U(K, J, Im) - U(K, Jp, Im))) / (dx_im * g2))
    u_div3 = ((rn_k * (U(K, J, I) - U(K, J, Im)) + rn_kp * (U(Kp, J, I) - U(Kp, J, Im))) /
              (dx_im * g3) +
              (rn_k * (V(K, J, I) - V(K, Jm, I)) + rn_kp * (V(Kp, J, I) - V(Kp, Jm, I))) /
              (dy_jm * g3))

    u_j_bar1 = 0.5 * dt * U(K, J, I) * (
        0.25 * (ra_k * W(K, J, Ip) + ra_k * W(K, J, I) + ra_km * W(Km, J, Ip) +
                ra_km * W(Km, J, I)) / g1 *
        (P(Kp, J, Ip) + P(Kp, J, I) - P(Km, J, Ip) - P(Km, J, I)) /
        (P(Kp, J, Ip) + P(Kp, J, I) + P(Km, J, Ip) + P(Km, J, I) + SMALL) /
        (0.5 * (dzn_km + dzn_k)) +
        0.25 * (rn_k * V(K, J, Ip) + rn_k * V(K, J, I) + rn_k * V(K, Jm, Ip) +
                rn_k * V(K, Jm, I)) / g1 *
        (P(K, Jp, Ip) + P(K, Jp, I) - P(K, Jm, Ip) - P(K, Jm, I)) /
        (P(K, Jp, Ip) + P(K, Jp, I) + P(K, Jm, Ip) + P(K, Jm, I) + SMALL) /
        (0.5 * (dyn_jm + dyn_j)))
    u_j_bar2 = 0.5 * dt * V(K, J, I) * (
        0.25 * (ra_k * W(K, Jp, I) + ra_k * W(K, J, I) + ra_km * W(Km, Jp, I) +
                ra_km * W(Km, J, I)) / g2 *
        (P(Kp, Jp, I) + P(Kp, J, I) - P(Km, Jp, I) - P(Km, J, I)) /
        (P(Kp, Jp, I) + P(Kp, J, I) + P(Km, Jp, I) + P(Km, J, I) + SMALL) /
        (0.5 * (dzn_km + dzn_k)) +
        0.25 * (rn_k * U(K, Jp, I) + rn_k * U(K, J, I) + rn_k * U(K, Jp, Im) +
                rn_k * U(K, J, Im)) / g2 *
        (P(K, Jp, Ip) + P(K, J, Ip) - P(K, Jp, Im) - P(K, J, Im)) /
        (P(K, Jp, Ip) + P(K, J, Ip) + P(K, Jp, Im) + P(K, J, Im) + SMALL) /
        (0.5 * (dxn_im + dxn_i)))
    u_j_bar3 = 0.5 * dt * W(K, J, I) * (
        0.25 * (rn_kp * V(Kp, J, I) + rn_k * V(K, J, I) + rn_kp * V(Kp, Jm, I) +
                rn_k * V(K, Jm, I)) / g3 *
        (P(Kp, Jp, I) + P(K, Jp, I) - P(Kp, Jm, I) - P(K, Jm, I)) /
        (P(Kp, Jp, I) + P(K, Jp, I) + P(Kp, Jm, I) + P(K, Jm, I) + SMALL) /
        (0.5 * (dyn_jm + dyn_j)) +
        0.25 * (rn_kp * U(Kp, J, I) + rn_k * U(K, J, I) + rn_kp * U(Kp, J, Im) +
                rn_k * U(K, J, Im)) / g3 *
        (P(Kp, J, Ip) + P(K, J, Ip) - P(Kp, J, Im) - P(K, J, Im)) /
        (P(Kp, J, Ip) + P(K, J, Ip) + P(Kp, J, Im) + P(K, J, Im) + SMALL) /
        (0.5 * (dxn_im + dxn_i)))

    uc, vc, wc = U(K, J, I), V(K, J, I), W(K, J, I)
    us_ = (np.abs(uc) * dx_i - dt * uc * uc) * (P(K, J, Ip) - P(K, J, I)) / \
        (P(K, J, Ip) + P(K, J, I) + SMALL) / dxn_i - u_j_bar1
    vs_ = (np.abs(vc) * dy_j - dt * vc * vc) * (P(K, Jp, I) - P(K, J, I)) / \
        (P(K, Jp, I) + P(K, J, I) + SMALL) / dyn_j - u_j_bar2
    ws_ = (np.abs(wc) * dz_k - dt * (ra_k / g3) * wc * wc) * (P(Kp, J, I) - P(K, J, I)) / \
        (P(Kp, J, I) + P(K, J, I) + SMALL) / dzn_k - u_j_bar3
    us[K, J, I] = us_ - 0.25 * dt * uc * ((U(K, J, Ip) - U(K, J, Im)) / dx_im + u_div1)
    vs[K, J, I] = vs_ - 0.25 * dt * vc * ((V(K, Jp, I) - V(K, Jm, I)) / dy_jm + u_div2)
    ws[K, J, I] = ws_ - 0.25 * dt * wc * ((ra_kp * W(Kp, J, I) - ra_km * W(Km, J, I)) /
                                          (dz_km * g3) + u_div3)


def _limited(g, dt, ut, vt, wt, psi, po, us, vs, ws):
    """us, vs, ws (interior): the FCT-limited velocities, :542-675."""
    kp = g.kp
    K, Km, Kp = slice(1, kp + 1), slice(0, kp), slice(2, kp + 2)
    J, Jm, Jp = slice(1, -1), slice(0, -2), slice(2, None)
    I, Im, Ip = slice(1, -1), slice(0, -2), slice(2, None)
    nb = [(K, J, I), (K, J, Im), (K, J, Ip), (K, Jm, I), (K, Jp, I), (Km, J, I), (Kp, J, I)]
    vals = [psi[s] for s in nb] + [po[s] for s in nb]
    pmax = np.maximum.reduce(vals)
    pmin = np.minimum.reduce(vals)
    ra, rn = _k(g.rhoa), _k(g.rhoan)
    rk, rkm = ra[K], ra[Km]
    rnk = rn[K]
    dxn, dyn, dzn = g.dxn[None, None, I], g.dyn[None, J, None], _k(g.dzn[K])
    p0 = po[K, J, I]
    mx, mn = np.maximum, np.minimum
    denom1 = dt * (
        (mx(ut[K, J, Im], 0.0) * rnk * po[K, J, Im] - mn(ut[K, J, I], 0.0) * rnk * po[K, J, Ip]) /
        dxn +
        (mx(vt[K, Jm, I], 0.0) * rnk * po[K, Jm, I] - mn(vt[K, J, I], 0.0) * rnk * po[K, Jp, I]) /
        dyn +
        (mx(wt[Km, J, I], 0.0) * rkm * po[Km, J, I] - mn(wt[K, J, I], 0.0) * rk * po[Kp, J, I]) /
        dzn) + SMALL
    denom2 = dt * (
        (mx(ut[K, J, I], 0.0) * rnk * p0 - mn(ut[K, J, Im], 0.0) * rnk * p0) / dxn +
        (mx(vt[K, J, I], 0.0) * rnk * p0 - mn(vt[K, Jm, I], 0.0) * rnk * p0) / dyn +
        (mx(wt[K, J, I], 0.0) * rk * p0 - mn(wt[Km, J, I], 0.0) * rkm * p0) / dzn + SMALL)
    bu = np.zeros_like(po, order="F")
    bd = np.zeros_like(po, order="F")
    bu[K, J, I] = rnk * (pmax - p0) / denom1
    bd[K, J, I] = rnk * (p0 - pmin) / denom2
    bicgstab_np.exchange_along_dim(bu, 0.0, 0.0)
    bicgstab_np.exchange_along_dim(bd, 0.0, 0.0)

    def m3(a, b, c):
        return np.minimum(np.minimum(a, b), c)

    one = 1.0
    us[K, J, I] = (m3(one, bd[K, J, I], bu[K, J, Ip]) * mx(ut[K, J, I], 0.0) +
                   m3(one, bu[K, J, I], bd[K, J, Ip]) * mn(ut[K, J, I], 0.0))
    vs[K, J, I] = (m3(one, bd[K, J, I], bu[K, Jp, I]) * mx(vt[K, J, I], 0.0) +
                   m3(one, bu[K, J, I], bd[K, Jp, I]) * mn(vt[K, J, I], 0.0))
    ws[K, J, I] = (m3(one, bd[K, J, I], bu[Kp, J, I]) * mx(wt[K, J, I], 0.0) +
                   m3(one, bu[K, J, I], bd[Kp, J, I]) * mn(wt[K, J, I], 0.0))


def _limited_sfvt(g, dt, ut, vt, wt, psi, po, us, vs, ws):
    """The limiter variant of sfvt/advection_3d.F90:544-704: bounds per
    direction from the three cells along it, no density weights, and
    dx(i-1), dy(j-1), dz(k-1) in the denominators."""
    kp = g.kp
    K, Km, Kp = slice(1, kp + 1), slice(0, kp), slice(2, kp + 2)
    J, Jm, Jp = slice(1, -1), slice(0, -2), slice(2, None)
    I, Im, Ip = slice(1, -1), slice(0, -2), slice(2, None)
    mx, mn = np.maximum, np.minimum

    def bounds(a, b, c):
        vals = [psi[a], psi[b], psi[c], po[a], po[b], po[c]]
        return np.maximum.reduce(vals), np.minimum.reduce(vals)
    C = (K, J, I)
    imax, imin = bounds((K, J, Im), C, (K, J, Ip))
    jmax, jmin = bounds((K, Jm, I), C, (K, Jp, I))
    kmax, kmin = bounds((Km, J, I), C, (Kp, J, I))
    dx, dy, dz = g.dx[None, None, Im], g.dy[None, Jm, None], _k(g.dz[Km])
    p0 = po[C]
    denom1 = (dt * ((mx(ut[K, J, Im], 0.0) * po[K, J, Im] - mn(ut[C], 0.0) * po[K, J, Ip]) / dx +
                    (mx(vt[K, Jm, I], 0.0) * po[K, Jm, I] - mn(vt[C], 0.0) * po[K, Jp, I]) / dy +
                    (mx(wt[Km, J, I], 0.0) * po[Km, J, I] - mn(wt[C], 0.0) * po[Kp, J, I]) / dz +
                    SMALL))
    denom2 = (dt * ((mx(ut[C], 0.0) * p0 - mn(ut[K, J, Im], 0.0) * p0) / dx +
                    (mx(vt[C], 0.0) * p0 - mn(vt[K, Jm, I], 0.0) * p0) / dy +
                    (mx(wt[C], 0.0) * p0 - mn(wt[Km, J, I], 0.0) * p0) / dz +
                    SMALL))
    beta = {}
    for name, hi, lo in (("i", imax, imin), ("j", jmax, jmin), ("k", kmax, kmin)):
        up = np.zeros_like(po, order="F")
        down = np.zeros_like(po, order="F")
        up[C] = (hi - p0) / denom1
        down[C] = (p0 - lo) / denom2
        bicgstab_np.exchange_along_dim(up, 0.0, 0.0)
        bicgstab_np.exchange_along_dim(down, 0.0, 0.0)
        beta[name] = (up, down)

    def m3(a, b, c):
        return np.minimum(np.minimum(a, b), c)
    (iu, idn), (ju, jdn), (ku, kdn) = beta["i"], beta["j"], beta["k"]
    us[C] = (m3(1.0, idn[C], iu[K, J, Ip]) * mx(ut[C], 0.0) +
             m3(1.0, iu[C], idn[K, J, Ip]) * mn(ut[C], 0.0))
    vs[C] = (m3(1.0, jdn[C], ju[K, Jp, I]) * mx(vt[C], 0.0) +
             m3(1.0, ju[C], jdn[K, Jp, I]) * mn(vt[C], 0.0))
    ws[C] = (m3(1.0, kdn[C], ku[Kp, J, I]) * mx(wt[C], 0.0) +
             m3(1.0, ku[C], kdn[Kp, J, I]) * mn(wt[C], 0.0))


def _mpdata(g, dt, u, v, w, fields, kord, monotone, neumann, bcs, limiter=0):
    """The passes of mpdata_3d / mpdata_vec_3d on shifted fields: the
    antidiffusive velocities and the limiter from fields[0], the donor cell
    and the exchange of every field with its (lbc, ubc) in bcs."""
    s1 = [np.zeros_like(u, order="F") for _ in range(3)]
    s2 = [np.zeros_like(u, order="F") for _ in range(3)]
    vel, sav = [u, v, w], s1
    psi = fields[0].copy(order="F") if kord > 1 else None
    po = fields[0]
    it2 = 0
    for it in range(1, kord + 1):
        if it > 1:
            it2 += 1
            _antidiffusive(g, dt, *vel, po, *sav)
            vel, sav = (s1, s2) if it2 % 2 == 1 else (s2, s1)
            for a in vel:
                cases.exchange_full(a, 0.0, 0.0)
        if it > 1 and monotone:
            it2 += 1
            (_limited_sfvt if limiter else _limited)(g, dt, *vel, psi, po, *sav)
            vel, sav = s2, s1
            for a in vel:
                cases.exchange_full(a, 0.0, 0.0)
        for f, (lb, ub) in zip(fields, bcs):
            dynamics_np.first_order_upstream_3d(g, dt, *vel, f, neumann)
            if it <= kord and kord >= 1:
                cases.exchange_full(f, lb, ub)


def mpdata_3d(g, dt, u, v, w, psi_in, lbc, ubc, kord, monotone, neumann=0, limiter=0):
    """psi_in advanced in place; returns the shifted-back (lbc, ubc).
    limiter = 1 takes the sfvt/ variant of the FCT limiter."""
    kp, jp, ip = g.kp, g.jp, g.ip
    mn = min(float(psi_in.min()), lbc, ubc)  # the whole array, halo included (:271)
    psi_in -= mn
    lbc -= mn
    ubc -= mn
    if float(np.sum(psi_in[1:kp + 1, 1:jp + 1, 1:ip + 1])) >= SMALL:
        _mpdata(g, dt, u, v, w, [psi_in], kord, monotone, neumann, [(lbc, ubc)], limiter)
    psi_in += mn
    return lbc + mn, ubc + mn


def mpdata_vec_3d(g, dt, u, v, w, fields, lbc, ubc, kord, monotone, neumann=0):
    """mpdata_vec_3d (advection_3d.F90:1250-1753): the fields of one category
    advanced in place with the velocities of the first; lbc, ubc (arrays)
    updated in place.  Each field is shifted by the minimum of its interior
    and its boundary values (:1299-1306)."""
    kp, jp, ip = g.kp, g.jp, g.ip
    mins = []
    for n, f in enumerate(fields):
        mn = min(float(f[1:kp + 1, 1:jp + 1, 1:ip + 1].min()), lbc[n], ubc[n])
        f -= mn
        lbc[n] -= mn
        ubc[n] -= mn
        mins.append(mn)
    if float(np.sum(fields[0][1:kp + 1, 1:jp + 1, 1:ip + 1])) >= SMALL:
        _mpdata(g, dt, u, v, w, fields, kord, monotone, neumann,
                [(lbc[n], ubc[n]) for n in range(len(fields))])
    for n, f in enumerate(fields):
        f += mins[n]
        lbc[n] += mins[n]
        ubc[n] += mins[n]


def mpdata_3d_add(g, dt, u, v, w, psi_in, psi_1d, lbc, ubc, kord, monotone, neumann=0):
    """mpdata_3d_add (advection_3d.F90:139-190): psi_1d(k) added to every level
    of the field (halo included), mpdata_3d, and subtracted again."""
    psi_in += psi_1d[:, None, None]
    lbc, ubc = mpdata_3d(g, dt, u, v, w, psi_in, lbc, ubc, kord, monotone, neumann)
    psi_in -= psi_1d[:, None, None]
    return lbc, ubc
