"""Array-at-a-time numpy restatements of five routines of the reference's time
step on one rank, independent checks of the oracle's C restatement:

* advance_momentum (dynamics.f90:1019-1099);
* divergence_calc (diagnostics.f90:120-153);
* adv_ref_state (pamm/sfvt/advection_3d.F90:1148-1218);
* first_order_upstream_3d (pamm/sfvt/advection_3d.F90:39-116);
* sources (dynamics.f90:639-1000): the centred momentum sources and
  buoyancy, damping, forcing and subsidence, the exchanges (or, with
  viscous = .true., the subgrid model), the boundary rows and the Poisson
  right-hand side.

Arrays are a(0:kp+1, 0:jp+1, 0:ip+1) in Fortran order, 1-D metrics
a(0:n+1).  Every expression keeps the reference's evaluation order (Fortran
evaluates operators of equal precedence left to right), so the results are
bit for bit the reference's arithmetic in IEEE double without fused
multiply-adds.
"""
import numpy as np

from helpers import cases

GRAV = 9.81  # dynamics.f90:18

I = slice(1, -1)  # interior along an axis


def _k(a):
    """a 1-D metric over levels as a (n, 1, 1) column"""
    return a[:, None, None]


def advance_momentum(g, dt, u, v, w, zu, zv, zw, su, sv, sw, p):
    """u, v, w at levels 0..kp of the interior columns, in place."""
    kp = g.kp
    K = slice(0, kp + 1)
    rn = _k(g.rhoan[K])
    u[K, I, I] = zu[K, I, I] + ((su[K, I, I] - (p[K, I, 2:] - p[K, I, I]) /
                                 g.dxn[None, None, 1:-1]) * dt) / rn
    v[K, I, I] = zv[K, I, I] + ((sv[K, I, I] - (p[K, 2:, I] - p[K, I, I]) /
                                 g.dyn[None, 1:-1, None]) * dt) / rn
    w[K, I, I] = zw[K, I, I] + ((sw[K, I, I] - (p[1:kp + 2, I, I] - p[K, I, I]) /
                                 _k(g.dzn[K])) * dt) / _k(g.rhoa[K])


def divergence_calc(g, u, v, w, div):
    """div at the interior points, in place."""
    rn = _k(g.rhoan[1:-1])
    div[I, I, I] = (rn * (u[I, I, I] - u[I, I, :-2]) / g.dx[None, None, :-2] +
                    rn * (v[I, I, I] - v[I, :-2, I]) / g.dy[None, :-2, None] +
                    (_k(g.rhoa[1:-1]) * w[I, I, I] - _k(g.rhoa[:-2]) * w[:-2, I, I]) /
                    _k(g.dz[:-2]))


def adv_ref_state(g, dt, w, psi, psi_ref):
    """psi at levels 1..kp of every column, halo columns included, in place."""
    kp = g.kp
    K, Km, Kp = slice(1, kp + 1), slice(0, kp), slice(2, kp + 2)
    pr = psi_ref
    psi[K] = psi[K] - dt * (0.5 / _k(g.dz[Km]) * w[Km] * _k(g.rhoa[Km]) * _k(pr[K] - pr[Km]) +
                            0.5 / _k(g.dz[K]) * w[K] * _k(g.rhoa[K]) * _k(pr[Kp] - pr[K])) / \
        _k(g.rhoan[K])


def first_order_upstream_3d(g, dt, u, v, w, psi, neumann=0):
    """Donor-cell update of psi at the interior points, in place."""
    dxn = g.dxn[None, None, 1:-1]
    dyn = g.dyn[None, 1:-1, None]
    dzn, ra, rn = _k(g.dzn[1:-1]), _k(g.rhoa), _k(g.rhoan[1:-1])
    c = psi[I, I, I]
    uc, ul = u[I, I, I], u[I, I, :-2]
    vc, vl = v[I, I, I], v[I, :-2, I]
    wc, wl = w[I, I, I], w[:-2, I, I]
    fx_r = ((uc + np.abs(uc)) * c + (uc - np.abs(uc)) * psi[I, I, 2:]) * dt / (2.0 * dxn)
    fx_l = ((ul + np.abs(ul)) * psi[I, I, :-2] + (ul - np.abs(ul)) * c) * dt / (2.0 * dxn)
    fy_r = ((vc + np.abs(vc)) * c + (vc - np.abs(vc)) * psi[I, 2:, I]) * dt / (2.0 * dyn)
    fy_l = ((vl + np.abs(vl)) * psi[I, :-2, I] + (vl - np.abs(vl)) * c) * dt / (2.0 * dyn)
    fz_r = ((wc + np.abs(wc)) * ra[1:-1] * c + (wc - np.abs(wc)) * ra[1:-1] * psi[2:, I, I]) * \
        dt / (2.0 * dzn * rn)
    fz_l = ((wl + np.abs(wl)) * ra[:-2] * psi[:-2, I, I] + (wl - np.abs(wl)) * ra[:-2] * c) * \
        dt / (2.0 * dzn * rn)
    if neumann == 1:
        fz_l[0] = fz_r[0]
        fz_r[-1] = fz_l[-1]
    elif neumann == 2:
        fz_l[0] = -fz_r[0]
        fz_r[-1] = -fz_l[-1]
    psi[I, I, I] = c - (fx_r - fx_l) - (fy_r - fy_l) - (fz_r - fz_l)


def sources(g, ubar, vbar, wbar, thbar, zu, zv, zw, u, v, w, th, su, sv, sw, sth, rhs,
            forcing=None, viscous=None):
    """su, sv, sw, sth and rhs in place.  viscous = dict(lamsq, z0, z0th, vism,
    vist, strain): viscous = .true., the subgrid model (tests/subgrid_np.py)
    in place of the four exchanges (dynamics.f90:878-893), with zeroed stress
    temporaries."""
    kp = g.kp
    K, Km, Kp = slice(1, kp + 1), slice(0, kp), slice(2, kp + 2)
    J, Jm, Jp = I, slice(0, -2), slice(2, None)
    Im, Ip = slice(0, -2), slice(2, None)
    rn, ra = _k(g.rhoan[K]), _k(g.rhoa[K])
    dx_i, dx_im = g.dx[None, None, I], g.dx[None, None, Im]
    dxn_i, dxn_im = g.dxn[None, None, I], g.dxn[None, None, Im]
    dy_j, dy_jm = g.dy[None, J, None], g.dy[None, Jm, None]
    dyn_j, dyn_jm = g.dyn[None, J, None], g.dyn[None, Jm, None]
    dz_k, dz_km = _k(g.dz[K]), _k(g.dz[Km])
    dzn_k, dzn_km = _k(g.dzn[K]), _k(g.dzn[Km])
    su[K, J, I] = rn * (
        (u[K, J, Im] * (u[K, J, I] + u[K, J, Im]) - u[K, J, Ip] * (u[K, J, I] + u[K, J, Ip])) /
        (2.0 * (dx_i + dx_im)) +
        (u[K, Jm, I] * (v[K, Jm, I] + v[K, Jm, Ip]) - u[K, Jp, I] * (v[K, J, I] + v[K, J, Ip])) /
        (2.0 * (dyn_j + dyn_jm)) +
        (u[Km, J, I] * (w[Km, J, I] + w[Km, J, Ip]) - u[Kp, J, I] * (w[K, J, I] + w[K, J, Ip])) /
        (2.0 * (dzn_k + dzn_km)))
    sv[K, J, I] = rn * (
        (v[K, J, Im] * (u[K, J, Im] + u[K, Jp, Im]) - v[K, J, Ip] * (u[K, J, I] + u[K, Jp, I])) /
        (2.0 * (dxn_i + dxn_im)) +
        (v[K, Jm, I] * (v[K, J, I] + v[K, Jm, I]) - v[K, Jp, I] * (v[K, J, I] + v[K, Jp, I])) /
        (2.0 * (dy_j + dy_jm)) +
        (v[Km, J, I] * (w[Km, J, I] + w[Km, Jp, I]) - v[Kp, J, I] * (w[K, J, I] + w[K, Jp, I])) /
        (2.0 * (dzn_k + dzn_km)))
    tb = thbar
    sw[K, J, I] = ra * (
        ((w[K, J, Im] * (u[K, J, Im] + u[Kp, J, Im]) - w[K, J, Ip] * (u[K, J, I] + u[Kp, J, I])) /
         (2.0 * (dxn_i + dxn_im)) +
         (w[K, Jm, I] * (v[K, Jm, I] + v[Kp, Jm, I]) - w[K, Jp, I] * (v[K, J, I] + v[Kp, J, I])) /
         (2.0 * (dyn_j + dyn_jm)) +
         (w[Km, J, I] * (w[K, J, I] + w[Km, J, I]) - w[Kp, J, I] * (w[K, J, I] + w[Kp, J, I])) /
         (2.0 * (dz_k + dz_km))) +
        GRAV * (th[K, J, I] + th[Kp, J, I]) /
        (2.0 * _k(g.theta[K]) + _k(tb[K]) + _k(tb[Kp])))
    f = forcing or {}
    if f.get("damping_layer"):
        dfn, df = _k(f["dampfacn"][K]), _k(f["dampfac"][K])
        su[K, J, I] = su[K, J, I] + rn * dfn * (zu[K, J, I] - _k(ubar[K]))
        sv[K, J, I] = sv[K, J, I] + rn * dfn * (zv[K, J, I] - _k(vbar[K]))
        sw[K, J, I] = sw[K, J, I] + ra * df * (zw[K, J, I] - 0.0)
        sth[K, J, I] = sth[K, J, I] + dfn * (th[K, J, I] - 0.0)
    if f.get("forcing"):
        tau = f.get("forcing_tau", 1.0)
        su[K, J, I] = su[K, J, I] - rn * (zu[K, J, I] - _k(f["u_force"][K])) / tau
        sv[K, J, I] = sv[K, J, I] - rn * (zv[K, J, I] - _k(f["v_force"][K])) / tau
    if f.get("divergence"):
        sw[K, J, I] = sw[K, J, I] - rn * (_k(wbar[K]) - _k(f["w_subs"][K]))
    if viscous:
        import subgrid_np

        vs = viscous
        taus = [np.zeros_like(su, order="F") for _ in range(6)]
        subgrid_np.subgrid(g, vs["lamsq"], vs["z0"], vs["z0th"], u, v, w, zu, zv, zw, th,
                           vs["vism"], vs["vist"], vs["strain"], taus, su, sv, sw, sth)
    else:
        for a in (su, sv, sw, sth):
            cases.exchange_full(a, 0.0, 0.0)
    su[0] = -su[1]
    sv[0] = -sv[1]
    sw[0] = 0.0
    sw[kp:kp + 2] = 0.0
    su[kp:kp + 2] = 0.0
    sv[kp:kp + 2] = 0.0
    K1, K1m = slice(1, kp + 2), slice(0, kp + 1)
    rhs[K1, J, I] = ((su[K1, J, I] - su[K1, J, Im]) / dx_im +
                     (sv[K1, J, I] - sv[K1, Jm, I]) / dy_jm +
                     (sw[K1, J, I] - sw[K1m, J, I]) / _k(g.dz[K1m]))
    rhs[0, J, I] = ((su[0, J, I] - su[0, J, Im]) / g.dx[None, Im] +
                    (sv[0, J, I] - sv[0, Jm, I]) / g.dy[Jm, None] +
                    (sw[0, J, I] + sw[1, J, I]) / g.dz[1])
