"""GPU parity of every per-call drop-in against the oracle, through the C-ABI.

Same seeded inputs on both sides; every halo cell is random on input so the
tests also pin which halo cells each routine reads and writes.  Copies and
exchanges must be bit-exact; arithmetic routines must agree to 1e-12 relative
max-norm per output field (the FP64 parity bar is 1e-10 after one time
step; single routines are held tighter).
"""
import numpy as np
import pytest

from helpers import (breakdown_system, breakdown_threshold, cases, fz, live_mask_p, rand_field,
                     relerr, small_bubble, velocities)

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module", params=["3d", "xz"])
def setup(request, dcm, orc):
    if request.param == "3d":
        c = small_bubble(ip=24, jp=20, kp=16)
    else:
        c = cases.kelvin_helmholtz(ip=40, jp=1, kp=12)
    g = c.grid
    core = dcm.DynamicalCore(g)
    ocore = orc.OracleCore(g)
    yield g, core, ocore
    core.close()


@pytest.mark.parametrize("kind", ["full", "dim", "wo"])
def test_exchange(setup, kind):
    g, core, ocore = setup
    rng = np.random.default_rng(10)
    a = rand_field(g, rng)
    b = a.copy(order="F")
    if kind == "full":
        core.exchange_full(a, 0.3, -0.7)
        ocore.exchange_full(b, 0.3, -0.7)
    elif kind == "dim":
        core.exchange_along_dim(a, 0.3, -0.7)
        ocore.exchange_along_dim(b, 0.3, -0.7)
        # vertical edges are untouched by both; compare everything
    else:
        core.exchange_along_dim_wo(a)
        ocore.exchange_along_dim_wo(b)
    assert np.array_equal(a, b)


def test_advance_momentum(setup):
    g, core, ocore = setup
    rng = np.random.default_rng(11)
    args = [rand_field(g, rng) for _ in range(10)]
    a2 = [x.copy(order="F") for x in args]
    core.advance_momentum(2.0, *args)
    ocore.advance_momentum(2.0, *a2)
    for x, y in zip(args[:3], a2[:3]):
        assert relerr(x, y) <= TOL


@pytest.mark.parametrize("damping", [False, True])
def test_sources(setup, damping):
    g, core, ocore = setup
    rng = np.random.default_rng(12)
    u, v, w = velocities(g, rng, 1.0)
    th = rand_field(g, rng, -0.5, 2.0)
    zu, zv, zw = (rand_field(g, rng) for _ in range(3))
    K2 = g.kp + 2
    bars = [rng.uniform(-1, 1, K2) for _ in range(4)]
    forcing = None
    if damping:
        forcing = dict(damping_layer=1, forcing=1, divergence=1,
                       dampfacn=rng.uniform(-0.01, 0, K2), dampfac=rng.uniform(-0.01, 0, K2),
                       u_force=rng.uniform(-1, 1, K2), v_force=rng.uniform(-1, 1, K2),
                       w_subs=rng.uniform(-0.01, 0.01, K2), forcing_tau=600.0)
    outs = [rand_field(g, rng) for _ in range(5)]  # su sv sw sth rhs (inout)
    outs2 = [o.copy(order="F") for o in outs]
    core.sources(*bars, zu, zv, zw, u, v, w, th, *outs, forcing=forcing)
    ocore.sources(*bars, zu, zv, zw, u, v, w, th, *outs2, forcing=forcing)
    for name, x, y in zip(("su", "sv", "sw", "sth", "rhs"), outs, outs2):
        assert relerr(x, y) <= TOL, name


@pytest.mark.parametrize("neumann", [0, 1, 2])
def test_first_order_upstream(setup, neumann):
    g, core, ocore = setup
    rng = np.random.default_rng(13)
    u, v, w = velocities(g, rng, 1.0)
    psi = rand_field(g, rng, 0.0, 1.0)
    p2 = psi.copy(order="F")
    core.first_order_upstream_3d(1.0, u, v, w, psi, neumann)
    ocore.first_order_upstream_3d(1.0, u, v, w, p2, neumann)
    assert relerr(psi, p2) <= TOL


@pytest.mark.parametrize("kord,monotone,neumann,limiter",
                         [(1, 1, 0, 0), (2, 1, 0, 0), (3, 1, 0, 0), (3, 0, 0, 0),
                          (3, 1, 1, 0), (3, 1, 2, 0), (3, 1, 0, 1), (4, 1, 0, 0)])
def test_mpdata_3d(setup, kord, monotone, neumann, limiter):
    g, core, ocore = setup
    rng = np.random.default_rng(14 + kord)
    u, v, w = velocities(g, rng, 1.0, courant=0.2)
    psi = rand_field(g, rng, -0.3, 1.0)  # random halos: min is over the whole array
    p2 = psi.copy(order="F")
    lb1, ub1 = core.mpdata_3d(1.0, u, v, w, psi, 0.1, -0.2, kord, monotone, neumann, limiter)
    lb2, ub2 = ocore.mpdata_3d(1.0, u, v, w, p2, 0.1, -0.2, kord, monotone, neumann, limiter)
    assert relerr(psi, p2) <= TOL
    assert lb1 == lb2 and ub1 == ub2


def test_mpdata_3d_early_return(setup):
    """A constant field shifts to all zeros: the sum test of :284-289 returns
    (psi - m) + m."""
    g, core, ocore = setup
    rng = np.random.default_rng(20)
    u, v, w = velocities(g, rng, 1.0, courant=0.2)
    psi = fz(g) + 0.3
    p2 = psi.copy(order="F")
    core.mpdata_3d(1.0, u, v, w, psi, 0.3, 0.3, 3, 1)
    ocore.mpdata_3d(1.0, u, v, w, p2, 0.3, 0.3, 3, 1)
    assert np.array_equal(psi, p2)


@pytest.mark.parametrize("limiter", [0, 1])
def test_mpdata_vec_3d(setup, dcm, limiter):
    g, core, ocore = setup
    rng = np.random.default_rng(21)
    u, v, w = velocities(g, rng, 1.0, courant=0.2)
    fields = [rand_field(g, rng, -0.2, 1.0) for _ in range(3)]
    q1 = dcm.fortran_stack(fields)
    q2 = dcm.fortran_stack(fields)
    lb1, ub1 = np.array([0.0, 0.1, -0.1]), np.array([0.0, 0.2, 0.05])
    lb2, ub2 = lb1.copy(), ub1.copy()
    core.mpdata_vec_3d(1.0, u, v, w, q1, lb1, ub1, 3, 1, 0, limiter)
    ocore.mpdata_vec_3d(1.0, u, v, w, q2, lb2, ub2, 3, 1, 0, limiter)
    for q in range(3):
        assert relerr(q1[q], q2[q]) <= TOL, q
    assert np.array_equal(lb1, lb2) and np.array_equal(ub1, ub2)


def test_adv_ref_state(setup):
    g, core, ocore = setup
    rng = np.random.default_rng(22)
    w = rand_field(g, rng)
    psi = rand_field(g, rng)
    p2 = psi.copy(order="F")
    core.adv_ref_state(1.0, w, psi, g.thetan)
    ocore.adv_ref_state(1.0, w, p2, g.thetan)
    assert relerr(psi, p2) <= TOL


def test_mpdata_3d_add(setup):
    g, core, ocore = setup
    rng = np.random.default_rng(23)
    u, v, w = velocities(g, rng, 1.0, courant=0.2)
    psi = rand_field(g, rng, -0.3, 1.0)
    p2 = psi.copy(order="F")
    r1 = core.mpdata_3d_add(1.0, u, v, w, psi, g.thetan, 299.0, 301.0, 3, 1)
    r2 = ocore.mpdata_3d_add(1.0, u, v, w, p2, g.thetan, 299.0, 301.0, 3, 1)
    assert relerr(psi, p2) <= TOL
    assert r1 == r2


def test_horizontal_means_and_divergence(setup, dcm):
    g, core, ocore = setup
    rng = np.random.default_rng(24)
    f = [rand_field(g, rng) for _ in range(4)]
    q = dcm.fortran_stack([rand_field(g, rng) for _ in range(2)])
    b1 = core.horizontal_means(*f, q=q)
    b2 = ocore.horizontal_means(*f, q=q)
    for x, y in zip(b1, b2):
        assert relerr(x, y) <= TOL
    d1 = rand_field(g, rng)
    d2 = d1.copy(order="F")
    core.divergence_calc(*f[:3], d1)
    ocore.divergence_calc(*f[:3], d2)
    assert relerr(d1, d2) <= TOL


def test_advance_scalar_fields(setup):
    g, core, ocore = setup
    rng = np.random.default_rng(25)
    th, sth = rand_field(g, rng), rand_field(g, rng)
    t2 = th.copy(order="F")
    core.advance_scalar_fields_3d(0.5, th, sth)
    ocore.advance_scalar_fields_3d(0.5, t2, sth)
    assert relerr(th, t2) <= TOL


def _poisson_rhs(g, rng):
    b = fz(g)
    b[1:-1, 1:-1, 1:-1] = rng.normal(size=(g.kp, g.jp, g.ip))
    b[1:-1, 1:-1, 1:-1] -= b[1:-1, 1:-1, 1:-1].mean()
    return b


def test_bicgstab(setup, orc, dcm):
    g, core, ocore = setup
    rng = np.random.default_rng(26)
    b = _poisson_rhs(g, rng)
    x = rand_field(g, rng, -0.01, 0.01)
    sw = rand_field(g, rng)
    x2, b2 = x.copy(order="F"), b.copy(order="F")
    it1, err1 = core.bicgstab(x, b, sw, 1e-10)
    st, it2, err2 = ocore.bicgstab(x2, b2, sw, 1e-10)
    assert st == 0
    assert it1 == it2
    assert err1 < 1e-10 and err2 < 1e-10
    # Both solves stop at ||r|| < tol * max(||b||, 0.01) (dynamics.f90:370-428),
    # so ||A (x1 - x2)|| <= 2 tol sc_err is what the algorithm guarantees;
    # the two runs differ only in dot-product summation order.
    d = x - x2
    ad = fz(g)
    ocore.mat_ax(np.asfortranarray(d), ad)
    sc = max(np.sqrt(np.sum(b[1:-1, 1:-1, 1:-1] ** 2)), 0.01)
    assert np.sqrt(np.sum(ad[1:-1, 1:-1, 1:-1] ** 2)) <= 2e-10 * sc
    ocore.exchange_along_dim_wo(x2)  # the driver's exchange after the solve
    m = live_mask_p(g)
    assert relerr(x, x2, m) <= 1e-9


def test_bicgstab_noconv_status(setup, dcm):
    g, core, ocore = setup
    rng = np.random.default_rng(27)
    b = _poisson_rhs(g, rng)
    with pytest.raises(dcm.DCMError) as e:
        core.bicgstab(fz(g), b, fz(g), 1e-10, itmax=1)
    assert e.value.status == dcm.DCM_E_NOCONV


def test_bicgstab_nonfinite_status(setup, dcm):
    g, core, ocore = setup
    rng = np.random.default_rng(28)
    b = _poisson_rhs(g, rng)
    b[3, 1, 2] = np.nan
    with pytest.raises(dcm.DCMError) as e:
        core.bicgstab(fz(g), b, fz(g), 1e-10)
    assert e.value.status == dcm.DCM_E_NONFINITE


def test_bicgstab_early_return(setup):
    """x already solves the system: the reference returns before the loop."""
    g, core, ocore = setup
    b = fz(g)
    x = fz(g) + 0.25
    x2 = x.copy(order="F")
    it, err = core.bicgstab(x, b.copy(order="F"), fz(g), 1e-10)
    st, it2, err2 = ocore.bicgstab(x2, b.copy(order="F"), fz(g), 1e-10)
    assert it == it2 == 0 and err == err2 == 0.0
    m = live_mask_p(g)
    assert np.array_equal(x[m], x2[m])


def _raw_bicgstab(core, x, b, sw, tol, itmax=9999):
    """dcm_bicgstab through ctypes, returning (status, iterations) without
    raising, so that a failure status and the iteration it came at are both
    visible."""
    import ctypes as C
    it = C.c_int(-1)
    err = C.c_double(0.0)
    st = core.lib.dcm_bicgstab(core.h, core.F(x), core.F(b), core.F(sw), float(tol), 0,
                               int(itmax), C.byref(it), C.byref(err))
    return st, it.value


@pytest.mark.parametrize("later", [False, True])
def test_bicgstab_breakdown_status(setup, orc, dcm, later):
    """The breakdown stop of dynamics.f90:414-417 (|omega| < tiny), reached on
    a well-posed system by raising the threshold on both sides: above every
    |omega| (the stop comes in iteration 1) or between the |omega| of a later
    iteration m and the smallest earlier one (the stop comes in iteration m).
    The oracle and the GPU stop in the same iteration with the breakdown
    status, before that iteration's x update."""
    import bicgstab_np

    g, core, ocore = setup
    b, x = breakdown_system(g)
    tiny, want_it = breakdown_threshold(bicgstab_np, g, x, b, later)
    x0 = x.copy(order="F")
    x2, b2 = x.copy(order="F"), b.copy(order="F")
    core.solver_limits(tiny=tiny)
    orc.set_breakdown_tiny(tiny)
    try:
        st, it = _raw_bicgstab(core, x, b.copy(order="F"), fz(g), 1e-10)
        st2, it2, _ = ocore.bicgstab(x2, b2, fz(g), 1e-10)
    finally:
        core.solver_limits()
        orc.set_breakdown_tiny(-1.0)
    assert st == dcm.DCM_E_BREAKDOWN and st2 == 2
    assert it == it2 == want_it
    inner = (slice(1, -1),) * 3
    if want_it == 1:
        assert np.array_equal(x[inner], x0[inner])
    else:
        assert relerr(x[inner], x2[inner]) <= 1e-9
    # the handle is usable afterwards and back on the reference's threshold
    it3, err3 = core.bicgstab(x, b.copy(order="F"), fz(g), 1e-10)
    assert err3 < 1e-10 and it3 > 1


@pytest.mark.parametrize("graphs", [1, 2])
def test_bicgstab_timeout_status(setup, dcm, graphs):
    """A graph-driven solve is bounded by its round budget: with a budget
    below the iterations the solve needs, the loop ends after exactly that
    many iterations with DCM_E_TIMEOUT (the device sets the status and the
    WHILE node's condition; nothing waits on the host), and the next solve
    with the default budget converges."""
    g, core, ocore = setup
    rng = np.random.default_rng(30)
    b = _poisson_rhs(g, rng)
    x = fz(g)
    core.solver_graphs(graphs)
    core.solver_limits(max_rounds=3)
    try:
        st, it = _raw_bicgstab(core, x, b.copy(order="F"), fz(g), 1e-10)
    finally:
        core.solver_limits()
        core.solver_graphs(1)
    assert st == dcm.DCM_E_TIMEOUT
    assert it == 3
    it2, err2 = core.bicgstab(fz(g), b.copy(order="F"), fz(g), 1e-10)
    assert err2 < 1e-10 and it2 > 3


def test_small_solver_matches_the_multi_kernel_solve(setup, dcm):
    """The one-cluster FP64 solve of small domains against the nine-kernel
    iteration on the same system: both stop at ||r|| < tol max(||b||, 0.01)
    (dynamics.f90:370-428), so ||A (x1 - x2)|| <= 2 tol sc_err, and only the
    dot products' summation order differs (iteration counts within three)."""
    g, core, ocore = setup
    rng = np.random.default_rng(31)
    b = _poisson_rhs(g, rng)
    x0 = rand_field(g, rng, -0.01, 0.01)
    sw = rand_field(g, rng)
    xs, xm = x0.copy(order="F"), x0.copy(order="F")
    try:
        core.set_small_solver(8192)
        its, errs = core.bicgstab(xs, b.copy(order="F"), sw, 1e-10)
        core.set_small_solver(0)
        itm, errm = core.bicgstab(xm, b.copy(order="F"), sw, 1e-10)
    finally:
        core.set_small_solver()
    assert errs < 1e-10 and errm < 1e-10
    assert abs(its - itm) <= 3, (its, itm)
    d = xs - xm
    ad = fz(g)
    ocore.mat_ax(np.asfortranarray(d), ad)
    sc = max(np.sqrt(np.sum(b[1:-1, 1:-1, 1:-1] ** 2)), 0.01)
    assert np.sqrt(np.sum(ad[1:-1, 1:-1, 1:-1] ** 2)) <= 2e-10 * sc
    m = live_mask_p(g)
    assert relerr(xs, xm, m) <= 1e-9
