"""An independent numpy restatement of the Smagorinsky subgrid model
(sgm/subgrid_3d.f90:38-493), written array-at-a-time, used only to
cross-check the C restatement in oracle/.  Fields are a[k, j, i] with halo 1
(shape (kp+2, jp+2, ip+2)); 1-D metrics are halo-inclusive."""
import math

import numpy as np

_pow_c = np.frompyfunc(math.pow, 2, 1)


def _pow(x, e):
    """x**e elementwise by the C library's pow"""
    return _pow_c(x, e).astype(np.float64)

PRN, SUBB, SUBC, SUBG, SUBH, SUBR, RIC = 0.95, 40.0, 16.0, 1.2, 0.0, 4.0, 0.25
GRAV, SMALL, KVON = 9.81, 1.e-10, 0.4
SUBA = 1.0 / PRN
SUBF = SUBA
RI_EPS = float(np.float32(1.e-15))  # a single-precision literal in the reference


def _exchange_dim_faces(a, kp, jp, ip, k0, k1):
    """periodic x faces then y faces over levels k0..k1"""
    a[k0:k1 + 1, 1:jp + 1, 0] = a[k0:k1 + 1, 1:jp + 1, ip]
    a[k0:k1 + 1, 1:jp + 1, ip + 1] = a[k0:k1 + 1, 1:jp + 1, 1]
    a[k0:k1 + 1, 0, 1:ip + 1] = a[k0:k1 + 1, jp, 1:ip + 1]
    a[k0:k1 + 1, jp + 1, 1:ip + 1] = a[k0:k1 + 1, 1, 1:ip + 1]


def exchange_full_wo(a):
    """every halo cell the periodic image of an interior cell, except the
    interior of planes 0 and kp+1, which keep their values"""
    kp, jp, ip = a.shape[0] - 2, a.shape[1] - 2, a.shape[2] - 2
    keep0 = a[0, 1:jp + 1, 1:ip + 1].copy()
    keep1 = a[kp + 1, 1:jp + 1, 1:ip + 1].copy()
    kk = np.r_[kp, 1:kp + 1, 1]
    jj = np.r_[jp, 1:jp + 1, 1]
    ii = np.r_[ip, 1:ip + 1, 1]
    a[...] = a[np.ix_(kk, jj, ii)]
    a[0, 1:jp + 1, 1:ip + 1] = keep0
    a[kp + 1, 1:jp + 1, 1:ip + 1] = keep1


def exchange_along_dim(a, lbc, ubc):
    kp, jp, ip = a.shape[0] - 2, a.shape[1] - 2, a.shape[2] - 2
    _exchange_dim_faces(a, kp, jp, ip, 1, kp)
    a[kp + 1] = ubc
    a[0] = lbc


def exchange_full(a, lbc, ubc):
    kp, jp, ip = a.shape[0] - 2, a.shape[1] - 2, a.shape[2] - 2
    kk = np.r_[kp, 1:kp + 1, 1]
    jj = np.r_[jp, 1:jp + 1, 1]
    ii = np.r_[ip, 1:ip + 1, 1]
    a[...] = a[np.ix_(kk, jj, ii)]
    a[kp + 1, 1:jp + 1, 1:ip + 1] = ubc
    a[0, 1:jp + 1, 1:ip + 1] = lbc


def subgrid(g, lamsq, z0, z0th, u, v, w, zu, zv, zw, th, vism, vist, strain, taus, su, sv, sw,
            sth, q=(), sq=()):
    """Updates vism, vist, strain, the six taus (tau11, tau22, tau33, tau12,
    tau13, tau23), su, sv, sw, sth and each sq in place."""
    kp, jp, ip = g.kp, g.jp, g.ip
    K, J, I = slice(1, kp + 1), slice(1, jp + 1), slice(1, ip + 1)

    def at(a, dk=0, dj=0, di=0):
        return a[1 + dk:kp + 1 + dk, 1 + dj:jp + 1 + dj, 1 + di:ip + 1 + di]

    def mk(m, d=0):
        return m[1 + d:kp + 1 + d][:, None, None]

    def mj(m, d=0):
        return m[1 + d:jp + 1 + d][None, :, None]

    def mi(m, d=0):
        return m[1 + d:ip + 1 + d][None, None, :]

    dx, dy, dz, dxn, dyn, dzn = g.dx, g.dy, g.dz, g.dxn, g.dyn, g.dzn
    t = ((at(u, 1) - at(u, 1, 0, -1)) / mi(dx, -1)) ** 2 + ((at(u) - at(u, 0, 0, -1)) / mi(dx, -1)) ** 2
    t = t + ((at(v, 1) - at(v, 1, -1)) / mj(dy, -1)) ** 2 + ((at(v) - at(v, 0, -1)) / mj(dy, -1)) ** 2
    t = t + ((at(w) - at(w, -1)) / mk(dz, -1)) ** 2 + ((at(w, 1) - at(w)) / mk(dz)) ** 2
    t = t + 0.5 * (((at(u, 1) - at(u)) / mk(dzn) + (at(w, 0, 0, 1) - at(w)) / mi(dxn)) ** 2 +
                   ((at(u, 1, 0, -1) - at(u, 0, 0, -1)) / mk(dz) +
                    (at(w) - at(w, 0, 0, -1)) / mi(dxn, -1)) ** 2)
    t = t + 0.5 * (((at(w) - at(w, 0, -1)) / mj(dyn, -1) + (at(v, 1, -1) - at(v, 0, -1)) / mk(dzn)) ** 2 +
                   ((at(w, 0, 1) - at(w)) / mj(dyn) + (at(v, 1) - at(v)) / mk(dzn)) ** 2)

    def s12(kk, di_u, di_v0, di_v1, jlo):
        # (du/dy + dv/dx) at level k+kk over the j-pair (jlo, jlo+1)
        return ((at(u, kk, jlo + 1, di_u) - at(u, kk, jlo, di_u)) / mj(dyn, jlo) +
                (at(v, kk, jlo, di_v1) - at(v, kk, jlo, di_v0)) / mi(dxn, di_v0)) ** 2

    terms = [s12(0, -1, -1, 0, -1), s12(0, -1, -1, 0, 0), s12(0, 0, 0, 1, -1), s12(0, 0, 0, 1, 0),
             s12(1, -1, -1, 0, -1), s12(0, -1, -1, 0, 0), s12(1, 0, 0, 1, -1), s12(1, 0, 0, 1, 0)]
    acc = terms[0]
    for x in terms[1:]:
        acc = acc + x
    t = t + 0.125 * acc
    strain[K, J, I] = t

    rip = GRAV * (at(th, 1) / mk(g.thetan, 1) - at(th) / mk(g.thetan)) / mk(dzn) / (t + RI_EPS)
    fm = np.zeros_like(rip)
    fh = np.zeros_like(rip)
    neg = rip < 0.0
    mid = (rip >= 0.0) & (rip < RIC)
    # real exponents (**0.5, **SUBR) through the C library's pow, as compiled
    # Fortran evaluates them (numpy's vectorised power may differ by an ulp)
    fm[neg] = _pow(1.0 - SUBC * rip[neg], 0.5)
    fh[neg] = SUBA * _pow(1.0 - SUBB * rip[neg], 0.5)
    fm[mid] = _pow(1.0 - rip[mid] / RIC, SUBR) * (1.0 - SUBH * rip[mid])
    fh[mid] = SUBF * _pow(1.0 - rip[mid] / RIC, SUBR) * (1.0 - SUBG * rip[mid])
    vism[K, J, I] = mk(lamsq) * np.sqrt(t) * fm
    vist[K, J, I] = mk(lamsq) * np.sqrt(t) * fh * mk(g.rhoa)
    vism[kp - 1:kp + 1] = 0.0
    vist[kp - 1:kp + 1] = 0.0

    z1 = g.z[1]
    u1, v1, th1 = u[1], v[1], th[1]
    vmag = 0.5 * np.sqrt((u1[J, I] + u1[J, 0:ip]) ** 2 + (v1[J, I] + v1[0:jp, I]) ** 2) + SMALL
    dth = th1[J, I] + g.thetan[1] - g.theta[0]
    rib = GRAV * dth * (z1 - z0) ** 2 / (g.theta[0] * vmag ** 2 * (z1 - z0th))
    lg = math.log(z1 / z0)
    kv2 = KVON ** 2
    gm = np.where(rib <= 0.0,
                  1.0 - 9.4 * rib / (1.0 + 70.0 * kv2 * np.sqrt(np.abs(rib * z1 / z0)) / lg ** 2),
                  1.0 / (1.0 + 4.7 * rib) ** 2)
    gh = np.where(rib <= 0.0,
                  1.0 - 9.4 * rib / (1.0 + 50.0 * kv2 * np.sqrt(np.abs(rib * z1 / z0)) / lg ** 2),
                  1.0 / (1.0 + 4.7 * rib) ** 2)
    ustar = KVON * vmag / lg * np.sqrt(gm)
    thstar = kv2 * vmag * dth / (ustar * PRN * lg ** 2) * gh
    vism[0, J, I] = ustar ** 2 * (z1 - z0) / vmag
    vist[0, J, I] = ustar * thstar / (dth / (z1 - z0th) + SMALL)
    exchange_full_wo(vism)
    exchange_full_wo(vist)

    t11, t22, t33, t12, t13, t23 = taus
    vm = at(vism) + at(vism, -1)
    t11[K, J, I] = mk(g.rhoan) * 1.0 * vm * (at(zu) - at(zu, 0, 0, -1)) / mi(dx, -1)
    t22[K, J, I] = mk(g.rhoan) * 1.0 * vm * (at(zv) - at(zv, 0, -1)) / mj(dy, -1)
    t33[K, J, I] = mk(g.rhoan) * 1.0 * vm * (at(zw) - at(zw, -1)) / mk(dz, -1)
    v8 = at(vism)
    for (a, b, c) in ((0, 1, 0), (-1, 0, 0), (-1, 1, 0), (0, 0, 1), (0, 1, 1), (-1, 0, 1), (-1, 1, 1)):
        v8 = v8 + at(vism, a, b, c)
    t12[K, J, I] = mk(g.rhoan) * 0.125 * v8 * ((at(zu, 0, 1) - at(zu)) / mj(dyn) +
                                                (at(zv, 0, 0, 1) - at(zv)) / mi(dxn))
    t13[K, J, I] = mk(g.rhoa) * 0.5 * (at(vism) + at(vism, 0, 0, 1)) * (
        (at(zu, 1) - at(zu)) / mk(dzn) + (at(zw, 0, 0, 1) - at(zw)) / mi(dxn))
    t23[K, J, I] = mk(g.rhoa) * 0.5 * (at(vism) + at(vism, 0, 1)) * (
        (at(zw, 0, 1) - at(zw)) / mj(dyn) + (at(zv, 1) - at(zv)) / mk(dzn))
    for a in taus:
        exchange_along_dim(a, 0.0, 0.0)

    Kw = slice(1, kp)       # k = 1..kp-1
    Ku = slice(2, kp)       # k = 2..kp-1

    def at2(a, ks, dk=0, dj=0, di=0):
        return a[ks.start + dk:ks.stop + dk, 1 + dj:jp + 1 + dj, 1 + di:ip + 1 + di]

    sw[Kw, J, I] = sw[Kw, J, I] + ((at2(t33, Kw, 1) - at2(t33, Kw)) / dzn[Kw][:, None, None] +
                                   (at2(t13, Kw) - at2(t13, Kw, 0, 0, -1)) / mi(dx, -1) +
                                   (at2(t23, Kw) - at2(t23, Kw, 0, -1)) / mj(dy, -1))
    su[Ku, J, I] = su[Ku, J, I] + ((at2(t11, Ku, 0, 0, 1) - at2(t11, Ku)) / mi(dxn) +
                                   (at2(t12, Ku) - at2(t12, Ku, 0, -1)) / mj(dy, -1) +
                                   (at2(t13, Ku) - at2(t13, Ku, -1)) / dz[1:kp - 1][:, None, None])
    sv[Ku, J, I] = sv[Ku, J, I] + ((at2(t22, Ku, 0, 1) - at2(t22, Ku)) / mj(dyn) +
                                   (at2(t12, Ku) - at2(t12, Ku, 0, 0, -1)) / mi(dx, -1) +
                                   (at2(t23, Ku) - at2(t23, Ku, -1)) / dz[1:kp - 1][:, None, None])
    for a in (su, sv, sw):
        exchange_full(a, 0.0, 0.0)

    def diffuse(s, ds):
        vt = vist
        xs = 0.25 * ((at(vt) + at(vt, 0, 0, -1) + at(vt, -1) + at(vt, -1, 0, -1)) *
                     (at(s, 0, 0, -1) - at(s)) / mi(dxn, -1) -
                     (at(vt, 0, 0, 1) + at(vt) + at(vt, -1, 0, 1) + at(vt, -1)) *
                     (at(s) - at(s, 0, 0, 1)) / mi(dxn)) / mi(dx, -1)
        ys = 0.25 * ((at(vt) + at(vt, 0, -1) + at(vt, -1) + at(vt, -1, -1)) *
                     (at(s, 0, -1) - at(s)) / mj(dyn, -1) -
                     (at(vt, 0, 1) + at(vt) + at(vt, -1, 1) + at(vt, -1)) *
                     (at(s) - at(s, 0, 1)) / mj(dyn)) / mj(dy, -1)
        zs = (at(vt, -1) * (at(s, -1) - at(s)) / mk(dz, -1) -
              at(vt) * (at(s) - at(s, 1)) / mk(dz)) / mk(dz, -1)
        ds[K, J, I] = ds[K, J, I] + (xs + ys + zs) / mk(g.rhoan)
        exchange_full(ds, 0.0, 0.0)

    diffuse(th, sth)
    for a, b in zip(q, sq):
        diffuse(a, b)
