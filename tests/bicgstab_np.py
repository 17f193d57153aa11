"""Array-at-a-time numpy restatement of the reference's pressure solve on one
rank, an independent check of the oracle's C restatement:

* set_mat_a (dynamics.f90:34-175): per-axis metric coefficients, a_c = 0 and
  a_p = 1 outside the interior (a_p = 1 and the others 0 first, :55-62);
* mat_ax (:187-229): exchange_along_dim(x, 0, 0), the Neumann rows
  x(0) = x(1), x(kp+1) = x(kp), then the 7-point sum in the reference's
  order;
* precondition (:241-270): s = r/a_p, then prit times s = s + (r - A s)/a_p,
  whole-array statements including the halo;
* bicgstab (:293-444) and inn_prod (:458-482).

Every expression keeps the reference's evaluation order, and inn_prod sums
in the Fortran loop order (k fastest, then j, then i) with a sequential
accumulate, so the result is bit for bit the reference's arithmetic in
IEEE double without fused multiply-adds.
"""
import math

import numpy as np

TINY = float(np.float32(1e-16))  # tiny = 1.e-16, a default-real literal (:321)
PRIT = 3                          # :322


def coefficients(g):
    """The interior coefficients as broadcastable arrays and the full a_p."""
    ip, jp, kp = g.ip, g.jp, g.kp
    i = np.arange(1, ip + 1)
    j = np.arange(1, jp + 1)
    k = np.arange(1, kp + 1)
    c = dict(
        ae=(1.0 / (g.dx[i - 1] * g.dxn[i]))[None, None, :],
        aw=(1.0 / (g.dx[i - 1] * g.dxn[i - 1]))[None, None, :],
        an=(1.0 / (g.dy[j - 1] * g.dyn[j]))[None, :, None],
        as_=(1.0 / (g.dy[j - 1] * g.dyn[j - 1]))[None, :, None],
        au=(1.0 / (g.dz[k - 1] * g.dzn[k]))[:, None, None],
        ad=(1.0 / (g.dz[k - 1] * g.dzn[k - 1]))[:, None, None],
    )
    ap = np.ones((kp + 2, jp + 2, ip + 2), order="F")
    ap[1:-1, 1:-1, 1:-1] = -c["ae"] - c["aw"] - c["an"] - c["as_"] - c["au"] - c["ad"]
    c["ap"] = ap
    return c


def exchange_along_dim(a, lbc, ubc):
    """Single rank: the x and y faces (levels 1..kp) take their periodic
    images, then the whole bottom and top planes take lbc and ubc."""
    kp, jp, ip = a.shape[0] - 2, a.shape[1] - 2, a.shape[2] - 2
    a[1:kp + 1, 1:jp + 1, 0] = a[1:kp + 1, 1:jp + 1, ip]
    a[1:kp + 1, 1:jp + 1, ip + 1] = a[1:kp + 1, 1:jp + 1, 1]
    a[1:kp + 1, 0, 1:ip + 1] = a[1:kp + 1, jp, 1:ip + 1]
    a[1:kp + 1, jp + 1, 1:ip + 1] = a[1:kp + 1, 1, 1:ip + 1]
    a[0, :, :] = lbc
    a[kp + 1, :, :] = ubc


def mat_ax(c, x):
    """A x; x's halo is set in place, as the reference's mat_ax does."""
    kp = x.shape[0] - 2
    exchange_along_dim(x, 0.0, 0.0)
    x[0, :, :] = x[1, :, :]
    x[kp + 1, :, :] = x[kp, :, :]
    ax = np.zeros_like(x, order="F")
    ax[1:-1, 1:-1, 1:-1] = (c["aw"] * x[1:-1, 1:-1, :-2] + c["ae"] * x[1:-1, 1:-1, 2:] +
                            c["as_"] * x[1:-1, :-2, 1:-1] + c["an"] * x[1:-1, 2:, 1:-1] +
                            c["ad"] * x[:-2, 1:-1, 1:-1] + c["au"] * x[2:, 1:-1, 1:-1] +
                            c["ap"][1:-1, 1:-1, 1:-1] * x[1:-1, 1:-1, 1:-1] + 0.0)
    return ax


def inn_prod(x, y):
    p = (x[1:-1, 1:-1, 1:-1] * y[1:-1, 1:-1, 1:-1]).ravel(order="F")
    return float(np.cumsum(p)[-1]) if p.size else 0.0


def precondition(c, r):
    s = r / c["ap"]
    for _ in range(PRIT):
        t = mat_ax(c, s)
        s = s + (r - t) / c["ap"]
    return s


def bicgstab(g, x, b, sw, tol, itmax=9999, tiny=TINY, trace=None):
    """Solve A x = b from the initial x (updated in place); returns
    (status, iterations, err) with status 0 (converged), 1 (no convergence
    within itmax) or 2 (|omega| < tiny).  trace: a list that receives omega
    of every iteration."""
    c = coefficients(g)
    kp = g.kp
    sc_err = max(math.sqrt(inn_prod(b, b)), 0.01)
    ax = mat_ax(c, x)
    r = b - ax
    cr = r.copy(order="F")
    p = np.zeros_like(x, order="F")
    v1 = np.zeros_like(x, order="F")
    err = math.sqrt(inn_prod(r, r)) / sc_err
    if err < tol:
        return 0, 0, err
    alf = omg = nrm = 1.0
    it = 0
    for it in range(1, itmax + 1):
        rho = inn_prod(r, cr)
        bet = (rho / nrm) * (alf / omg)
        t = r - bet * (omg * v1)
        s = precondition(c, t)
        p = s + bet * p
        v1 = mat_ax(c, p)
        nrm = inn_prod(cr, v1)
        alf = rho / nrm
        s = r - alf * v1
        cs = precondition(c, s)
        t = mat_ax(c, cs)
        tt = inn_prod(t, t)
        ts = inn_prod(t, s)
        omg = ts / tt
        if trace is not None:
            trace.append(omg)
        if abs(omg) < tiny:
            return 2, it, err
        x[...] = x + alf * p + omg * cs
        r = s - omg * t
        err = math.sqrt(inn_prod(r, r)) / sc_err
        nrm = rho
        if err < tol:
            break
    if err > tol:
        return 1, it, err
    x[kp + 1, :, :] = x[kp, :, :]
    x[0, :, :] = x[1, :, :] - sw[0, :, :] * g.dzn[0]
    return 0, it, err
