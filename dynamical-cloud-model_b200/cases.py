"""Seeded synthetic inputs for the dynamical core (stand-in for allocate_and_set).

The reference builds its grid, hydrostatic base state and initial fields in
``allocate_and_set`` (initialisation.f90:117-888) from a namelist and a
sounding.  The workloads measured here have no reference namelist, so this
module builds the same arrays directly:

* grid (initialisation.f90:428-446): uniform spacings; x(i) = dx*i -
  (ip-1)/2*dx, xn = x - dx/2 (same for y); z(k) = k*dz, zn = z - dz/2, for the
  halo-inclusive index range 0..n+1;
* base state: hydrostatic balance dp/dz = -g p / (Ra T), T = theta (p/1e5)^(Ra/cp)
  (hydrostatic1a, initialisation.f90:1475-1506) integrated exactly through the
  Exner function, d(pi)/dz = -g/(cp theta), for a piecewise-linear theta
  sounding; rho = p / (Ra theta (p/1e5)^(Ra/cp)) on z (rhoa, theta) and zn
  (rhoan, thetan) levels (:511-578);
* winds on zn levels with u = v = 0 for k <= 1 and k = kp (:757-808); the
  three time levels start equal; u, v, w and theta get exchange_full(0, 0)
  (:862-871);
* perturbations: numpy PCG64 with the seed stated per case.

Every field is a numpy array of shape (kp+2, jp+2, ip+2) in Fortran order, the
reference's own memory layout a(0:kp+1, 0:jp+1, 0:ip+1).
"""
from dataclasses import dataclass, field
import math

import numpy as np

RA, CP, GRAV = 287.0, 1005.0, 9.81  # initialisation.f90:9


def fzeros(kp, jp, ip):
    return np.zeros((kp + 2, jp + 2, ip + 2), dtype=np.float64, order="F")


@dataclass
class Grid:
    ip: int
    jp: int
    kp: int
    dx: np.ndarray
    dxn: np.ndarray
    dy: np.ndarray
    dyn: np.ndarray
    dz: np.ndarray
    dzn: np.ndarray
    rhoa: np.ndarray
    rhoan: np.ndarray
    theta: np.ndarray
    thetan: np.ndarray
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    xn: np.ndarray
    yn: np.ndarray
    zn: np.ndarray

    @property
    def shape(self):
        return (self.kp + 2, self.jp + 2, self.ip + 2)

    @property
    def npoints(self):
        return self.ip * self.jp * self.kp


def exchange_full(a, lbc=0.0, ubc=0.0):
    """Single-rank exchange_full (mpi_module.f90:926-1271): every halo cell is
    the periodic image of an interior cell except the interior of the top and
    bottom planes, which hold ubc / lbc."""
    kp, jp, ip = a.shape[0] - 2, a.shape[1] - 2, a.shape[2] - 2
    kk = np.r_[kp, 1:kp + 1, 1]
    jj = np.r_[jp, 1:jp + 1, 1]
    ii = np.r_[ip, 1:ip + 1, 1]
    a[...] = a[np.ix_(kk, jj, ii)]
    a[kp + 1, 1:jp + 1, 1:ip + 1] = ubc
    a[0, 1:jp + 1, 1:ip + 1] = lbc
    return a


def mixing_length_sq(grid, cvis=0.23, z0=1.0e-4):
    """Smagorinsky mixing length squared on the w-levels, lamsq
    (initialisation.f90:449-450), with the nominal horizontal spacings taken
    from the grid's first interior cells.  cvis = 0.23 and z0 = 1e-4 m are
    the reference's namelist.in values."""
    dx_nm, dy_nm = float(grid.dx[1]), float(grid.dy[1])
    return 1.0 / (1.0 / (cvis * (dx_nm + dy_nm + grid.dz) / 3.0) ** 2.0 +
                  1.0 / (0.4 * (grid.z + z0)) ** 2.0)


def _interp(zs, ths, z):
    """Linear interpolation of the sounding with the reference's clamps:
    find_pos / poly_int over the bracketing pair, min(z, z_top)."""
    zz = np.minimum(z, zs[-1])
    idx = np.clip(np.searchsorted(zs, zz, side="right") - 1, 0, len(zs) - 2)
    z0, z1 = zs[idx], zs[idx + 1]
    t0, t1 = ths[idx], ths[idx + 1]
    return t0 + (t1 - t0) * (zz - z0) / (z1 - z0)


def _inv_theta_integral(zs, ths, z):
    """Integral of 1/theta(z') from 0 to z for the piecewise-linear sounding
    (exact per segment: log for a sloped segment, linear for a flat one)."""
    out = np.zeros_like(z)
    for n, zt in enumerate(z):
        lo, hi = (0.0, zt) if zt >= 0 else (zt, 0.0)
        sign = 1.0 if zt >= 0 else -1.0
        knots = np.concatenate(([lo], zs[(zs > lo) & (zs < hi)], [hi]))
        tot = 0.0
        for a, b in zip(knots[:-1], knots[1:]):
            ta, tb = _interp(zs, ths, np.array([a, b]))
            if abs(tb - ta) < 1e-14 * abs(ta):
                tot += (b - a) / ta
            else:
                tot += (b - a) * math.log(tb / ta) / (tb - ta)
        out[n] = sign * tot
    return out


def make_grid(ip, jp, kp, dx, dy, dz, sounding_z, sounding_theta, psurf=1.0e5):
    idx_i = np.arange(ip + 2, dtype=np.float64)
    idx_j = np.arange(jp + 2, dtype=np.float64)
    idx_k = np.arange(kp + 2, dtype=np.float64)
    x = dx * idx_i - (ip - 1) / 2.0 * dx
    y = dy * idx_j - (jp - 1) / 2.0 * dy
    z = dz * idx_k
    xn, yn, zn = x - 0.5 * dx, y - 0.5 * dy, z - 0.5 * dz
    zs = np.asarray(sounding_z, dtype=np.float64)
    ts = np.asarray(sounding_theta, dtype=np.float64)
    kappa = RA / CP
    pis = (psurf / 1.0e5) ** kappa

    def state(levels):
        th = _interp(zs, ts, levels)
        exner = pis - GRAV / CP * _inv_theta_integral(zs, ts, levels)
        p = 1.0e5 * exner ** (1.0 / kappa)
        rho = p / (RA * th * (p / 1.0e5) ** kappa)
        return th, rho

    theta, rhoa = state(z)
    thetan, rhoan = state(zn)
    full = lambda n, v: np.full(n + 2, float(v))
    return Grid(ip, jp, kp, full(ip, dx), full(ip, dx), full(jp, dy), full(jp, dy),
                full(kp, dz), full(kp, dz), rhoa, rhoan, theta, thetan, x, y, z, xn, yn, zn)


@dataclass
class State:
    """Fields handed to model_driver: velocities in the roles current (u),
    previous (zu) and next (tu), and the scalars."""
    u: np.ndarray
    v: np.ndarray
    w: np.ndarray
    zu: np.ndarray
    zv: np.ndarray
    zw: np.ndarray
    tu: np.ndarray
    tv: np.ndarray
    tw: np.ndarray
    th: np.ndarray
    p: np.ndarray
    q: np.ndarray = None  # (nq, kp+2, jp+2, ip+2) stacked, each Fortran ordered
    extra: dict = field(default_factory=dict)

    def copy(self):
        def cp(a):
            if a is None:
                return None
            if isinstance(a, list):
                return [x.copy(order="K") for x in a]
            return a.copy(order="K")
        c = State(**{k: cp(getattr(self, k))
                     for k in ("u", "v", "w", "zu", "zv", "zw", "tu", "tv", "tw", "th", "p",
                               "q")})
        c.extra = dict(self.extra)
        return c


def _winds(g, ufun, vfun=None):
    u = fzeros(g.kp, g.jp, g.ip)
    v = fzeros(g.kp, g.jp, g.ip)
    uz = ufun(g.zn)
    vz = vfun(g.zn) if vfun else np.zeros_like(g.zn)
    uz[g.kp] = 0.0
    vz[g.kp] = 0.0
    uz[:2] = 0.0
    vz[:2] = 0.0
    u[...] = uz[:, None, None]
    v[...] = vz[:, None, None]
    return u, v


def _state(g, u, v, th, nq=0, q=None):
    w = fzeros(g.kp, g.jp, g.ip)
    zu, zv, zw = u.copy(order="F"), v.copy(order="F"), w.copy(order="F")
    tu, tv, tw = u.copy(order="F"), v.copy(order="F"), w.copy(order="F")
    for a in (u, v, w, th):
        exchange_full(a, 0.0, 0.0)
    if q is not None:
        exchange_full(q[0], 0.0, 0.0)
    return State(u, v, w, zu, zv, zw, tu, tv, tw, th, fzeros(g.kp, g.jp, g.ip), q)


# ---------------------------------------------------------------------------
# the workloads
# ---------------------------------------------------------------------------

@dataclass
class Case:
    name: str
    grid: Grid
    state: State
    dt: float
    nsteps: int
    kord: int
    monotone: int = 1
    ptol: float = 1e-10
    nq: int = 0
    ncat: int = 0
    c_s: tuple = ()
    c_e: tuple = ()
    seed: int = 0


def kelvin_helmholtz(ip=128, jp=1, kp=64, seed=1):
    """2-D x-z dry shear layer: dx = dz = 20 m, u = 10 tanh((zn-640)/50),
    theta 300 K below 640 m and 302 K above (the sounding is given at every
    zn level), theta' ~ U(-0.1, 0.1) K; dt = 0.5 s, 600 steps, kord = 2."""
    dx = dz = 20.0
    zn = dz * np.arange(kp + 2) - 0.5 * dz
    ths = np.where(zn < 640.0, 300.0, 302.0)
    g = make_grid(ip, jp, kp, dx, dx, dz, zn, ths)
    u, v = _winds(g, lambda z: 10.0 * np.tanh((z - 640.0) / 50.0))
    rng = np.random.Generator(np.random.PCG64(seed))
    th = fzeros(kp, jp, ip)
    th[1:kp + 1, 1:jp + 1, 1:ip + 1] = rng.uniform(-0.1, 0.1, size=(kp, jp, ip))
    return Case("kelvin_helmholtz_%dx%dx%d" % (ip, jp, kp), g, _state(g, u, v, th), 0.5, 600,
                kord=2, seed=seed)


def warm_bubble(ip=256, jp=256, kp=128, dxyz=50.0, amp=2.0, radius=1000.0, zc=1500.0,
                sigma=0.01, seed=2, dt=1.0, nsteps=100):
    """3-D dry warm bubble at rest: theta = 300 K, +amp * cos^2(pi r / (2R))
    for r <= R = 1 km centred at (0, 0, 1500 m), plus seeded N(0, sigma) noise;
    dt = 1 s, 100 steps, kord = 3 (two antidiffusive iterations), monotone."""
    g = make_grid(ip, jp, kp, dxyz, dxyz, dxyz, [-1.0e4, 1.0e5], [300.0, 300.0])
    u, v = _winds(g, lambda z: np.zeros_like(z))
    rng = np.random.Generator(np.random.PCG64(seed))
    th = fzeros(kp, jp, ip)
    X = g.xn[None, None, 1:ip + 1]
    Y = g.yn[None, 1:jp + 1, None]
    Z = g.zn[1:kp + 1, None, None]
    r = np.sqrt(X * X + Y * Y + (Z - zc) ** 2)
    bub = np.where(r <= radius, amp * np.cos(np.pi * r / (2.0 * radius)) ** 2, 0.0)
    th[1:kp + 1, 1:jp + 1, 1:ip + 1] = bub + rng.normal(0.0, sigma, size=(kp, jp, ip))
    return Case("warm_bubble_%dx%dx%d" % (ip, jp, kp), g, _state(g, u, v, th), dt, nsteps,
                kord=3, seed=seed)


def sheared_convection(ip=512, jp=512, kp=256, ntracers=8, seed=4):
    """3-D sheared convection: dx = dy = dz = 25 m, u = 5 zn / 6400 m/s,
    theta' ~ U(-0.5, 0.5) K below 500 m, 8 passive tracers ~ U[0, 1], each its
    own category; dt = 0.5 s, 50 steps, kord = 3."""
    d = 25.0
    g = make_grid(ip, jp, kp, d, d, d, [-1.0e4, 1.0e5], [300.0, 300.0])
    u, v = _winds(g, lambda z: 5.0 * z / 6400.0)
    rng = np.random.Generator(np.random.PCG64(seed))
    th = fzeros(kp, jp, ip)
    low = (g.zn[1:kp + 1] < 500.0)
    th[1:kp + 1, 1:jp + 1, 1:ip + 1] = np.where(
        low[:, None, None], rng.uniform(-0.5, 0.5, size=(kp, jp, ip)), 0.0)
    qs = []
    for n in range(ntracers):
        a = fzeros(kp, jp, ip)
        a[1:kp + 1, 1:jp + 1, 1:ip + 1] = rng.uniform(0.0, 1.0, size=(kp, jp, ip))
        exchange_full(a, 0.0, 0.0)
        qs.append(a)
    st = _state(g, u, v, th)
    st.q = qs
    return Case("sheared_convection_%dx%dx%d" % (ip, jp, kp), g, st, 0.5, 50, kord=3,
                nq=ntracers, ncat=ntracers, c_s=tuple(range(1, ntracers + 1)),
                c_e=tuple(range(1, ntracers + 1)), seed=seed)


def ensemble_members(n=64, seed=5):
    """Sizes and amplitudes of the batched warm-bubble ensemble: ip, jp from
    {64, 96, 128, 192}, kp from {48, 64, 96}, amplitude U(1, 3) K."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for m in range(n):
        ip = int(rng.choice([64, 96, 128, 192]))
        jp = int(rng.choice([64, 96, 128, 192]))
        kp = int(rng.choice([48, 64, 96]))
        amp = float(rng.uniform(1.0, 3.0))
        out.append((ip, jp, kp, amp, seed * 1000 + m))
    return out
