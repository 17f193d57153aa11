"""Seeded inputs and comparison helpers shared by the tests."""
import numpy as np

from conftest import load_dcm

dcm = load_dcm()
cases = __import__("dcm_b200.cases", fromlist=["cases"])


def fz(g):
    return np.zeros((g.kp + 2, g.jp + 2, g.ip + 2), order="F")


def rand_field(g, rng, lo=-1.0, hi=1.0):
    """Random values in every cell, halos included (the routines must read
    the halos they are given)."""
    a = fz(g)
    a[...] = rng.uniform(lo, hi, size=a.shape)
    return a


def velocities(g, rng, dt, courant=0.35):
    """Random velocities with |u| dt/dx <= courant, halos exchanged."""
    u, v, w = fz(g), fz(g), fz(g)
    for a, d in ((u, g.dx[1]), (v, g.dy[1]), (w, g.dz[1])):
        a[...] = rng.uniform(-1.0, 1.0, size=a.shape) * courant * d / dt
        cases.exchange_full(a, 0.0, 0.0)
    w[0] = 0.0
    w[g.kp + 1] = 0.0
    return u, v, w


def relerr(a, b, mask=None):
    a = np.asarray(a)
    b = np.asarray(b)
    if mask is not None:
        a = a[mask]
        b = b[mask]
    den = np.max(np.abs(b))
    num = np.max(np.abs(a - b))
    if den == 0.0:
        return num
    return num / den


def live_mask_p(g):
    """Cells of p that the reference computes and later reads: everything
    except the halo rings of the top/bottom rows and the vertical halo edges,
    which hold solver residue in the reference and are never read."""
    m = np.ones((g.kp + 2, g.jp + 2, g.ip + 2), dtype=bool, order="F")
    jh = np.zeros(g.jp + 2, dtype=bool)
    jh[[0, g.jp + 1]] = True
    ih = np.zeros(g.ip + 2, dtype=bool)
    ih[[0, g.ip + 1]] = True
    ring = jh[:, None] | ih[None, :]
    m[0][ring] = False
    m[g.kp + 1][ring] = False
    edge = jh[:, None] & ih[None, :]
    m[1:g.kp + 1][:, edge] = False
    return m


def small_bubble(ip=24, jp=20, kp=16, seed=7, dxyz=100.0):
    return cases.warm_bubble(ip=ip, jp=jp, kp=kp, dxyz=dxyz, radius=500.0, zc=800.0,
                             seed=seed)


def subgrid_inputs(g, seed):
    """Seeded inputs of the subgrid model: winds of a few m/s and potential
    temperature perturbations of a few kelvin (so that both Richardson
    branches and both surface-layer branches occur), every halo cell set;
    the inout fields random too (the routine must keep what it does not
    write)."""
    rng = np.random.default_rng(seed)
    f = {n: rand_field(g, rng, -4.0, 4.0) for n in ("u", "v", "w", "zu", "zv", "zw")}
    f["th"] = rand_field(g, rng, -3.0, 3.0)
    for n in ("vism", "vist", "strain", "tau11", "tau22", "tau33", "tau12", "tau13", "tau23",
              "su", "sv", "sw", "sth"):
        f[n] = rand_field(g, rng, -1.0, 1.0)
    return f


def breakdown_system(g, seed=14):
    """A zero-mean Poisson right-hand side and a small random warm start."""
    rng = np.random.default_rng(seed)
    b = fz(g)
    b[1:-1, 1:-1, 1:-1] = rng.normal(size=(g.kp, g.jp, g.ip))
    b[1:-1, 1:-1, 1:-1] -= b[1:-1, 1:-1, 1:-1].mean()
    return b, rand_field(g, rng, -0.01, 0.01)


def breakdown_threshold(bicgstab_np, g, x0, b, later, n=12):
    """A breakdown threshold and the iteration it stops the solve in.  Not
    later: far above any |omega| (iteration 1).  later: the geometric mean of
    |omega_m| and the smallest earlier |omega|, for the first iteration m > 1
    whose |omega| is below every earlier one (omega from the numpy
    restatement of the reference's solve); the gap is far wider than the
    round-off between implementations."""
    if not later:
        return 1e300, 1
    trace = []
    bicgstab_np.bicgstab(g, x0.copy(order="F"), b.copy(order="F"), fz(g), 1e-30, itmax=n,
                         tiny=0.0, trace=trace)
    om = [abs(w) for w in trace]
    for m in range(1, len(om)):
        lo = min(om[:m])
        if om[m] < lo * (1 - 1e-4):
            return float(np.sqrt(om[m] * lo)), m + 1
    raise AssertionError("no iteration with a new smallest |omega| in the first %d" % n)
