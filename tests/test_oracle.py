"""CPU tests of the oracle (the CPU restatement the GPU tests compare with).

Parity with the Fortran reference is unpinned (no compiler for it here and no
golden vectors in it); these tests pin the restatement to independent
restatements and to analytic invariants instead.
"""
import numpy as np
import pytest

from helpers import (breakdown_system, breakdown_threshold, cases, fz, rand_field, relerr,
                     small_bubble, subgrid_inputs, velocities)


@pytest.fixture(scope="module")
def g():
    return small_bubble().grid


def test_exchange_full_matches_independent_restatement(orc, g):
    rng = np.random.default_rng(0)
    a = rand_field(g, rng)
    b = a.copy(order="F")
    orc.OracleCore(g).exchange_full(a, 0.25, -0.5)
    cases.exchange_full(b, 0.25, -0.5)
    assert np.array_equal(a, b)


def test_exchange_along_dim_rows_and_faces(orc, g):
    rng = np.random.default_rng(1)
    a = rand_field(g, rng)
    ref = a.copy(order="F")
    orc.OracleCore(g).exchange_along_dim(a, 3.0, 4.0)
    kp, jp, ip = g.kp, g.jp, g.ip
    assert np.all(a[0] == 3.0) and np.all(a[kp + 1] == 4.0)
    assert np.array_equal(a[1:kp + 1, 1:jp + 1, 0], ref[1:kp + 1, 1:jp + 1, ip])
    assert np.array_equal(a[1:kp + 1, 0, 1:ip + 1], ref[1:kp + 1, jp, 1:ip + 1])
    # vertical edges untouched
    assert np.array_equal(a[1:kp + 1, 0, 0], ref[1:kp + 1, 0, 0])


def test_mpdata_keeps_constant_in_nondivergent_flow(orc, g):
    """u(z), v(z), w = 0 is non-divergent: a constant tracer must stay
    constant through kord = 3 monotone MPDATA."""
    rng = np.random.default_rng(2)
    o = orc.OracleCore(g)
    u, v, w = fz(g), fz(g), fz(g)
    prof = rng.uniform(-3, 3, size=g.kp + 2)
    u[...] = prof[:, None, None]
    v[...] = -prof[:, None, None]
    psi = fz(g) + 1.7
    lb, ub = o.mpdata_3d(1.0, u, v, w, psi, 1.7, 1.7, 3, True)
    assert np.max(np.abs(psi - 1.7)) < 1e-13
    assert lb == 1.7 and ub == 1.7


def test_mpdata_conserves_mass(orc, g):
    """Periodic x, y and w = 0 at the bottom and top faces: sum rhoan*psi is
    conserved to round-off by the donor cell and the antidiffusive passes."""
    rng = np.random.default_rng(3)
    o = orc.OracleCore(g)
    u, v, w = velocities(g, rng, 1.0)
    w[g.kp] = 0.0
    psi = rand_field(g, rng, 0.0, 1.0)
    cases.exchange_full(psi, 0.0, 0.0)
    m0 = np.sum(g.rhoan[1:-1, None, None] * psi[1:-1, 1:-1, 1:-1])
    o.mpdata_3d(1.0, u, v, w, psi, 0.0, 0.0, 3, True)
    m1 = np.sum(g.rhoan[1:-1, None, None] * psi[1:-1, 1:-1, 1:-1])
    assert abs(m1 - m0) / abs(m0) < 1e-12


def test_mpdata_monotone_bounds(orc, g):
    """The FCT limiter keeps the result inside the range spanned by the input
    and its donor-cell update (the flow is divergent, so the donor cell may
    itself exceed the input range); without the limiter it overshoots."""
    rng = np.random.default_rng(4)
    o = orc.OracleCore(g)
    u, v, w = velocities(g, rng, 1.0, courant=0.2)
    psi = fz(g)
    psi[1:-1, 1:-1, 1:-1] = (rng.uniform(size=(g.kp, g.jp, g.ip)) > 0.7).astype(float)
    cases.exchange_full(psi, 0.0, 0.0)
    up = psi.copy(order="F")
    o.first_order_upstream_3d(1.0, u, v, w, up)
    lo = min(psi.min(), up[1:-1, 1:-1, 1:-1].min())
    hi = max(psi.max(), up[1:-1, 1:-1, 1:-1].max())
    free = psi.copy(order="F")
    o.mpdata_3d(1.0, u, v, w, psi, 0.0, 0.0, 3, True)
    assert psi.min() >= lo - 1e-12 and psi.max() <= hi + 1e-12
    o.mpdata_3d(1.0, u, v, w, free, 0.0, 0.0, 3, False)
    assert free.max() > hi or free.min() < lo


def test_bicgstab_manufactured_solution(orc, g):
    """b = A p* for a smooth p* obeying the Neumann rows; the solve from zero
    must reproduce p* up to the null space (a constant) within tolerance."""
    o = orc.OracleCore(g)
    kp, jp, ip = g.kp, g.jp, g.ip
    X = 2 * np.pi * np.arange(ip + 2) / ip
    Y = 2 * np.pi * np.arange(jp + 2) / jp
    Z = np.pi * (np.arange(kp + 2) - 0.5) / kp
    ps = np.asfortranarray(np.cos(Z)[:, None, None] * np.cos(X)[None, None, :] *
                           (1 + 0.5 * np.sin(Y))[None, :, None])
    b = fz(g)
    o.mat_ax(ps.copy(order="F"), b)
    x = fz(g)
    sw = fz(g)
    st, it, err = o.bicgstab(x, b, sw, 1e-10)
    assert st == 0 and err < 1e-10 and it > 0
    d = x[1:-1, 1:-1, 1:-1] - ps[1:-1, 1:-1, 1:-1]
    d -= d.mean()
    assert np.max(np.abs(d)) < 1e-6 * np.max(np.abs(ps))


@pytest.mark.parametrize("stretched", [False, True])
def test_bicgstab_matches_independent_restatement(orc, g, stretched):
    """The oracle's solve against an array-at-a-time numpy restatement of
    set_mat_a, mat_ax, precondition, bicgstab and inn_prod
    (tests/bicgstab_np.py): the same iterations and the same pressure, halo
    included, bit for bit.  A warm start from a random x; on the stretched
    grid every coefficient table varies along its axis."""
    import dataclasses

    import bicgstab_np

    rng = np.random.default_rng(11)
    if stretched:
        def spacing(n, d):
            return d * rng.uniform(0.7, 1.4, size=n + 2)
        g = dataclasses.replace(g, dx=spacing(g.ip, 100.0), dxn=spacing(g.ip, 100.0),
                                dy=spacing(g.jp, 100.0), dyn=spacing(g.jp, 100.0),
                                dz=spacing(g.kp, 80.0), dzn=spacing(g.kp, 80.0))
    o = orc.OracleCore(g)
    kp, jp, ip = g.kp, g.jp, g.ip
    X = 2 * np.pi * np.arange(ip + 2) / ip
    Z = np.pi * (np.arange(kp + 2) - 0.5) / kp
    ps = np.asfortranarray(np.cos(Z)[:, None, None] * np.sin(X)[None, None, :] *
                           (1 + rng.uniform(-0.3, 0.3, size=(1, jp + 2, 1))))
    b = fz(g)
    o.mat_ax(ps.copy(order="F"), b)
    x0 = rand_field(g, rng, -0.5, 0.5)
    sw = rand_field(g, rng, -0.1, 0.1)
    x_c, x_np = x0.copy(order="F"), x0.copy(order="F")
    st, it, err = o.bicgstab(x_c, b.copy(order="F"), sw, 1e-10)
    st2, it2, err2 = bicgstab_np.bicgstab(g, x_np, b.copy(order="F"), sw, 1e-10)
    assert (st, it) == (st2, it2) and st == 0 and it > 5
    assert err == err2
    assert np.array_equal(x_c, x_np)


def test_bicgstab_itmax_reports_noconv(orc, g):
    rng = np.random.default_rng(5)
    o = orc.OracleCore(g)
    b = fz(g)
    b[1:-1, 1:-1, 1:-1] = rng.normal(size=(g.kp, g.jp, g.ip))
    b[1:-1, 1:-1, 1:-1] -= b[1:-1, 1:-1, 1:-1].mean()
    st, it, err = o.bicgstab(fz(g), b, fz(g), 1e-10, itmax=1)
    assert st == 1 and it == 1 and err > 1e-10


@pytest.mark.parametrize("later", [False, True])
def test_bicgstab_breakdown_stop(orc, g, later):
    """The breakdown stop (dynamics.f90:414-417): with the threshold raised
    above |omega|, the solve stops in that iteration with status 2 before the
    iteration's x update, as the numpy restatement does.  later: the
    threshold sits between |omega| of the first iteration m > 1 that is
    smaller than every earlier one and the smallest earlier one, so the stop
    comes in iteration m after m - 1 full iterations."""
    import bicgstab_np

    b, x0 = breakdown_system(g)
    tiny, want_it = breakdown_threshold(bicgstab_np, g, x0, b, later)
    o = orc.OracleCore(g)
    x_c, x_np = x0.copy(order="F"), x0.copy(order="F")
    orc.set_breakdown_tiny(tiny)
    try:
        st, it, err = o.bicgstab(x_c, b.copy(order="F"), fz(g), 1e-10)
    finally:
        orc.set_breakdown_tiny(-1.0)
    st2, it2, err2 = bicgstab_np.bicgstab(g, x_np, b.copy(order="F"), fz(g), 1e-10, tiny=tiny)
    assert (st, it) == (st2, it2) == (2, want_it)
    assert np.array_equal(x_c, x_np)
    inner = (slice(1, -1),) * 3
    assert np.array_equal(x_c[inner], x0[inner]) == (want_it == 1)


def test_horizontal_means_match_numpy(orc, g):
    """Level means against numpy: to round-off against numpy's own mean, and
    bit for bit against the reference's sequential sum
    (driver_np.horizontal_means)."""
    import driver_np

    rng = np.random.default_rng(6)
    f = [rand_field(g, rng) for _ in range(4)]
    bars = orc.OracleCore(g).horizontal_means(*f)
    for a, bar in zip(f, bars[:4]):
        ref = a[:, 1:-1, 1:-1].mean(axis=(1, 2))
        assert relerr(bar, ref) < 1e-14
        assert np.array_equal(bar, driver_np.horizontal_means(a))


def test_step_projection_is_divergence_free(orc):
    """After a step the rho-weighted divergence of the new velocity is at the
    level of the solver tolerance (the pressure projection works)."""
    c = small_bubble()
    m = orc.OracleModel(c.grid, c.state, c.dt, ptol=c.ptol, kord=c.kord)
    m.driver_start()
    m.step(2)
    f = m.fields()
    div = fz(c.grid)
    m.core.divergence_calc(f["u"], f["v"], f["w"], div)
    rho_u = np.max(np.abs(f["w"])) * np.max(c.grid.rhoa) / c.grid.dz[1]
    assert np.max(np.abs(div[1:-1, 1:-1, 1:-1])) < 1e-6 * rho_u


def test_step_kh_2d_runs(orc):
    c = cases.kelvin_helmholtz(ip=32, jp=1, kp=16)
    m = orc.OracleModel(c.grid, c.state, c.dt, ptol=c.ptol, kord=c.kord)
    m.driver_start()
    it, err = m.step(3)
    assert it > 0 and err < 1e-10
    f = m.fields()
    assert np.all(np.isfinite(f["u"])) and np.all(np.isfinite(f["th"]))


def test_exchange_full_wo_matches_independent_restatement(orc, g):
    import subgrid_np
    rng = np.random.default_rng(5)
    a = rand_field(g, rng)
    b = a.copy(order="F")
    orc.OracleCore(g).exchange_full_wo(a)
    subgrid_np.exchange_full_wo(b)
    assert np.array_equal(a, b)


def test_subgrid_matches_independent_restatement(orc, g):
    """calculate_subgrid_3d: the C restatement against the array-at-a-time
    numpy one, every output field bit for bit, moisture on (two q fields)."""
    import subgrid_np
    lamsq = cases.mixing_length_sq(g, 0.23, 0.1)
    a = subgrid_inputs(g, 21)
    rng = np.random.default_rng(22)
    qs = [rand_field(g, rng, 0.0, 1e-2) for _ in range(2)]
    sqs = [rand_field(g, rng, -1e-5, 1e-5) for _ in range(2)]
    b = {n: x.copy(order="F") for n, x in a.items()}
    _fortran_stack = orc._fortran_stack
    q = _fortran_stack(qs)
    sq = _fortran_stack(sqs)
    viss = _fortran_stack([fz(g), fz(g)])
    orc.OracleCore(g).calculate_subgrid_3d(
        lamsq, 0.1, 0.1, a["u"], a["v"], a["w"], a["zu"], a["zv"], a["zw"], a["th"], a["vism"],
        a["vist"], a["strain"], a["tau11"], a["tau22"], a["tau33"], a["tau12"], a["tau13"],
        a["tau23"], a["su"], a["sv"], a["sw"], a["sth"], q=q, viss=viss, sq=sq)
    sq_np = [x.copy(order="F") for x in sqs]
    subgrid_np.subgrid(g, lamsq, 0.1, 0.1, b["u"], b["v"], b["w"], b["zu"], b["zv"], b["zw"],
                       b["th"], b["vism"], b["vist"], b["strain"],
                       [b[n] for n in ("tau11", "tau22", "tau33", "tau12", "tau13", "tau23")],
                       b["su"], b["sv"], b["sw"], b["sth"], q=qs, sq=sq_np)
    for n in a:
        assert np.array_equal(a[n], b[n]), n
    for m in range(2):
        assert np.array_equal(sq[m], sq_np[m]), m
        assert np.array_equal(viss[m], a["vist"]), m
    # both branches of the Richardson functions and a live surface layer
    kp = g.kp
    assert np.any(a["vism"][1:kp - 1] == 0.0) and np.any(a["vism"][1:kp - 1] > 0.0)
    assert np.all(np.isfinite(a["vism"][0, 1:-1, 1:-1]))


def _stretched(g, rng):
    import dataclasses

    def spacing(n, d):
        return d * rng.uniform(0.7, 1.4, size=n + 2)
    return dataclasses.replace(g, dx=spacing(g.ip, 100.0), dxn=spacing(g.ip, 100.0),
                               dy=spacing(g.jp, 100.0), dyn=spacing(g.jp, 100.0),
                               dz=spacing(g.kp, 80.0), dzn=spacing(g.kp, 80.0),
                               rhoa=rng.uniform(0.8, 1.2, size=g.kp + 2),
                               rhoan=rng.uniform(0.8, 1.2, size=g.kp + 2),
                               theta=rng.uniform(295.0, 305.0, size=g.kp + 2))


def test_step_routines_match_independent_restatement(orc, g):
    """advance_momentum, divergence_calc, adv_ref_state and
    first_order_upstream_3d (all three neumann modes) against array-at-a-time
    numpy restatements (tests/dynamics_np.py), bit for bit over the whole
    arrays, on a grid with varying spacings and densities."""
    import dynamics_np as dn

    rng = np.random.default_rng(12)
    g = _stretched(g, rng)
    o = orc.OracleCore(g)
    f = {n: rand_field(g, rng) for n in ("u", "v", "w", "zu", "zv", "zw", "su", "sv", "sw", "p")}
    a = {n: f[n].copy(order="F") for n in ("u", "v", "w")}
    b = {n: f[n].copy(order="F") for n in ("u", "v", "w")}
    rest = [f[n] for n in ("zu", "zv", "zw", "su", "sv", "sw", "p")]
    o.advance_momentum(0.7, a["u"], a["v"], a["w"], *rest)
    dn.advance_momentum(g, 0.7, b["u"], b["v"], b["w"], *rest)
    for n in ("u", "v", "w"):
        assert np.array_equal(a[n], b[n]), n
        assert not np.array_equal(a[n], f[n]), n  # the routine wrote something

    d1 = rand_field(g, rng)
    d0, d2 = d1.copy(order="F"), d1.copy(order="F")
    o.divergence_calc(f["u"], f["v"], f["w"], d1)
    dn.divergence_calc(g, f["u"], f["v"], f["w"], d2)
    assert np.array_equal(d1, d2) and not np.array_equal(d1, d0)

    ref = rng.uniform(290.0, 310.0, size=g.kp + 2)
    p1 = rand_field(g, rng)
    p0, p2 = p1.copy(order="F"), p1.copy(order="F")
    o.adv_ref_state(0.9, f["w"], p1, ref)
    dn.adv_ref_state(g, 0.9, f["w"], p2, ref)
    assert np.array_equal(p1, p2) and not np.array_equal(p1, p0)

    u, v, w = velocities(g, rng, 1.0)
    for neumann in (0, 1, 2):
        q1 = rand_field(g, rng, 0.0, 2.0)
        q0, q2 = q1.copy(order="F"), q1.copy(order="F")
        o.first_order_upstream_3d(1.0, u, v, w, q1, neumann)
        dn.first_order_upstream_3d(g, 1.0, u, v, w, q2, neumann)
        assert np.array_equal(q1, q2) and not np.array_equal(q1, q0), neumann


@pytest.mark.parametrize("kord,monotone,neumann,limiter",
                         [(1, False, 0, 0), (2, False, 0, 0), (3, False, 1, 0), (2, True, 0, 0),
                          (3, True, 0, 0), (3, True, 2, 0), (2, True, 0, 1), (3, True, 1, 1)])
def test_mpdata_matches_independent_restatement(orc, g, kord, monotone, neumann, limiter):
    """mpdata_3d against an array-at-a-time numpy restatement
    (tests/mpdata_np.py): the advected field, halo included, and the shifted
    boundary values, bit for bit, on a grid with varying spacings and
    densities and with random winds (halos included)."""
    import mpdata_np

    rng = np.random.default_rng(13 + kord + 10 * neumann + (100 if monotone else 0) +
                                1000 * limiter)
    g = _stretched(g, rng)
    o = orc.OracleCore(g)
    u, v, w = velocities(g, rng, 0.4)
    psi = rand_field(g, rng, -0.5, 2.0)
    p1, p2 = psi.copy(order="F"), psi.copy(order="F")
    winds = [a.copy(order="F") for a in (u, v, w)]
    lb1, ub1 = o.mpdata_3d(0.8, u, v, w, p1, 0.3, -0.7, kord, monotone, neumann, limiter)
    lb2, ub2 = mpdata_np.mpdata_3d(g, 0.8, u, v, w, p2, 0.3, -0.7, kord, monotone, neumann,
                                   limiter)
    assert (lb1, ub1) == (lb2, ub2)
    assert np.array_equal(p1, p2) and not np.array_equal(p1, psi)
    for a, b in zip((u, v, w), winds):
        assert np.array_equal(a, b)  # the winds are inputs only


@pytest.mark.parametrize("damping", [False, True])
def test_sources_match_independent_restatement(orc, g, damping):
    """sources with viscous = .false. against an array-at-a-time numpy
    restatement (tests/dynamics_np.py), with damping, forcing and subsidence
    off and on: su, sv, sw, sth and the Poisson right-hand side, halos and
    rows included, bit for bit."""
    import dynamics_np as dn

    rng = np.random.default_rng(14 + damping)
    g = _stretched(g, rng)
    o = orc.OracleCore(g)
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
    outs2 = [a.copy(order="F") for a in outs]
    o.sources(*bars, zu, zv, zw, u, v, w, th, *outs, forcing=forcing)
    dn.sources(g, *bars, zu, zv, zw, u, v, w, th, *outs2, forcing=forcing)
    for name, x, y in zip(("su", "sv", "sw", "sth", "rhs"), outs, outs2):
        assert np.array_equal(x, y), name


def test_driver_step_matches_independent_restatement(orc):
    """Three dry time steps of the oracle's model_driver (every phase of the
    u, zu, tu rotation) against the numpy restatement of the step
    (tests/driver_np.py), which chains the numpy restatements of its
    routines: every field, role and level mean, halos included, bit for
    bit, and the same iterations."""
    import driver_np

    c = small_bubble(ip=12, jp=10, kp=8)
    m = orc.OracleModel(c.grid, c.state, c.dt, ptol=c.ptol, kord=c.kord, monotone=c.monotone)
    d = driver_np.Driver(c.grid, c.state, c.dt, ptol=c.ptol, kord=c.kord, monotone=c.monotone)
    m.driver_start()
    d.start()
    for n in range(3):
        it, err = m.step(1)
        d.step()
        assert (it, err) == (d.iters, d.err), n
        a, b = m.fields(), d.fields()
        for name in b:
            assert np.array_equal(a[name], b[name]), (n, name)


@pytest.mark.parametrize("kord,monotone", [(2, False), (3, True)])
def test_mpdata_vec_matches_independent_restatement(orc, g, kord, monotone):
    """mpdata_vec_3d (a category of 3 fields advected with the velocities and
    bounds of its first) against the numpy restatement
    (tests/mpdata_np.py): every field, halo included, and the boundary
    values, bit for bit."""
    import mpdata_np

    rng = np.random.default_rng(31 + kord)
    g = _stretched(g, rng)
    o = orc.OracleCore(g)
    u, v, w = velocities(g, rng, 0.4)
    fields = [rand_field(g, rng, lo, 2.0) for lo in (-0.5, 0.0, 1.0)]
    stack = orc._fortran_stack(fields)
    mine = [f.copy(order="F") for f in fields]
    lb1, ub1 = np.array([0.3, 0.0, 1.5]), np.array([-0.7, 0.2, 1.1])
    lb2, ub2 = lb1.copy(), ub1.copy()
    o.mpdata_vec_3d(0.8, u, v, w, stack, lb1, ub1, kord, monotone)
    mpdata_np.mpdata_vec_3d(g, 0.8, u, v, w, mine, lb2, ub2, kord, monotone)
    assert np.array_equal(lb1, lb2) and np.array_equal(ub1, ub2)
    for q in range(3):
        assert np.array_equal(stack[q], mine[q]), q
        assert not np.array_equal(mine[q], fields[q]), q


def test_mpdata_add_matches_independent_restatement(orc, g):
    """mpdata_3d_add (advection scheme 2) against the numpy restatement: the
    field and the boundary values, bit for bit."""
    import mpdata_np

    rng = np.random.default_rng(41)
    g = _stretched(g, rng)
    o = orc.OracleCore(g)
    u, v, w = velocities(g, rng, 0.4)
    psi = rand_field(g, rng, -0.5, 0.5)
    prof = np.linspace(300.0, 330.0, g.kp + 2)
    p1, p2 = psi.copy(order="F"), psi.copy(order="F")
    b1 = o.mpdata_3d_add(0.8, u, v, w, p1, prof, 0.2, -0.1, 3, True)
    b2 = mpdata_np.mpdata_3d_add(g, 0.8, u, v, w, p2, prof, 0.2, -0.1, 3, True)
    assert b1 == b2
    assert np.array_equal(p1, p2) and not np.array_equal(p1, psi)


def test_driver_step_with_tracers_matches_independent_restatement(orc):
    """Two time steps of the oracle's model_driver with three passive q
    categories (the tracer configuration's path: mpdata_vec_3d per category,
    advance_scalar_fields_3d) against the numpy restatement: every field,
    each q, bit for bit."""
    import driver_np

    c = cases.sheared_convection(ip=12, jp=10, kp=8, ntracers=3)
    kw = dict(ptol=c.ptol, kord=c.kord, monotone=c.monotone)
    m = orc.OracleModel(c.grid, c.state, c.dt, nq=c.nq, c_s=c.c_s, c_e=c.c_e, **kw)
    d = driver_np.Driver(c.grid, c.state, c.dt, c_s=c.c_s, c_e=c.c_e, **kw)
    m.driver_start()
    d.start()
    for n in range(2):
        it, err = m.step(1)
        d.step()
        assert (it, err) == (d.iters, d.err), n
        a, b = m.fields(), d.fields()
        for name in b:
            if name == "q":
                for q in range(3):
                    assert np.array_equal(a["q"][q], b["q"][q]), (n, q)
            else:
                assert np.array_equal(a[name], b[name]), (n, name)


def test_viscous_sources_match_independent_restatement(orc, g):
    """sources with viscous = .true. (the subgrid model in place of the
    exchanges) against the numpy restatements: su, sv, sw, sth, the
    right-hand side, vism, vist and strain bit for bit."""
    import dynamics_np as dn

    rng = np.random.default_rng(51)
    o = orc.OracleCore(g)
    a = subgrid_inputs(g, 52)
    lamsq = cases.mixing_length_sq(g, 0.23, 0.1)
    bars = [rng.uniform(-1, 1, g.kp + 2) for _ in range(3)] + [rng.uniform(-0.5, 0.5, g.kp + 2)]
    outs = [rand_field(g, rng) for _ in range(5)]  # su sv sw sth rhs
    outs2 = [x.copy(order="F") for x in outs]
    vis1 = {n: fz(g) for n in ("vism", "vist", "strain")}
    vis2 = {n: fz(g) for n in ("vism", "vist", "strain")}
    o.sources_viscous(*bars, a["zu"], a["zv"], a["zw"], a["u"], a["v"], a["w"], a["th"], *outs,
                      lamsq, 0.1, 0.1, vis1["vism"], vis1["vist"], vis1["strain"])
    dn.sources(g, *bars, a["zu"], a["zv"], a["zw"], a["u"], a["v"], a["w"], a["th"], *outs2,
               viscous=dict(lamsq=lamsq, z0=0.1, z0th=0.1, **vis2))
    for name, x, y in zip(("su", "sv", "sw", "sth", "rhs"), outs, outs2):
        assert np.array_equal(x, y), name
    for n in vis1:
        assert np.array_equal(vis1[n], vis2[n]) and np.any(vis1[n]), n


def test_viscous_driver_step_matches_independent_restatement(orc):
    """Three viscous time steps of the oracle's model_driver against the
    numpy driver with the subgrid model in sources: every field, role, mean
    and the subgrid fields, bit for bit."""
    import driver_np

    c = small_bubble(ip=12, jp=10, kp=8)
    vis = dict(lamsq=cases.mixing_length_sq(c.grid, 0.23, 0.1), z0=0.1, z0th=0.1)
    kw = dict(ptol=c.ptol, kord=c.kord, monotone=c.monotone, viscous=vis)
    m = orc.OracleModel(c.grid, c.state, c.dt, **kw)
    d = driver_np.Driver(c.grid, c.state, c.dt, **kw)
    m.driver_start()
    d.start()
    for n in range(3):
        it, err = m.step(1)
        d.step()
        assert (it, err) == (d.iters, d.err), n
        a, b = m.fields(), d.fields()
        for name in b:
            ref = m.f[name] if name in ("vism", "vist", "strain") else a[name]
            assert np.array_equal(ref, b[name]), (n, name)
