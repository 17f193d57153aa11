"""GPU checks of the mixed-precision form (precision=1): FP32 fields and FP32
BiCGSTAB iterations with FP64 reliable updates of the FP64 pressure.

The oracle runs the reference's FP64 step on the same inputs; the mixed form
differs from it by FP32 round-off carried through the step and the solve.
Bars (relative max-norm against the oracle): MIXED_TOL for every field and
for p on its live cells.  The pressure still converges to ptol on the FP64
residual ||b - A p|| / max(||b||, 0.01) (dynamics.f90:370-428), which the
tests check through the reported error.
"""
import numpy as np
import pytest

from helpers import cases, live_mask_p, relerr, small_bubble

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-5
FIELDS = ("u", "v", "w", "zu", "zv", "zw", "th", "su", "sv", "sw")


def _run(dcm, orc, c, nsteps, precond=0, **kw):
    core = dcm.DynamicalCore(c.grid)
    core.upload_state(c.state, c.dt, ptol=c.ptol, kord=c.kord, monotone=c.monotone,
                      nq=c.nq, c_s=c.c_s, c_e=c.c_e, precision=1, precond=precond, **kw)
    core.driver_start()
    errs = []
    for _ in range(nsteps):
        errs.append(core.step(1).err_last)
    got = core.download_state()
    core.close()
    m = orc.OracleModel(c.grid, c.state, c.dt, ptol=c.ptol, kord=c.kord, monotone=c.monotone,
                        nq=c.nq, c_s=c.c_s, c_e=c.c_e, **kw)
    m.driver_start()
    for _ in range(nsteps):
        m.step(1)
    return got, m.fields(), errs


def _errors(c, got, ref):
    e = {n: relerr(got[n], ref[n]) for n in FIELDS}
    e["p"] = relerr(got["p"], ref["p"], live_mask_p(c.grid))
    return e


# The 2-D shear layer is held to one step: its u of 10 m/s makes the centred
# momentum sources near-cancelling sums, which FP32 fields resolve to about
# 1e-3 of their own size after a few steps (whatever the preconditioner).
@pytest.mark.parametrize("case,nsteps,precond", [("bubble", 1, 0), ("kh", 1, 0), ("bubble", 10, 0),
                                                 ("bubble", 10, 1), ("kh", 1, 1)])
def test_mixed_against_oracle(dcm, orc, case, nsteps, precond):
    c = small_bubble() if case == "bubble" else cases.kelvin_helmholtz(ip=40, jp=1, kp=12)
    got, ref, errs = _run(dcm, orc, c, nsteps, precond=precond)
    assert all(e < c.ptol for e in errs), errs
    e = _errors(c, got, ref)
    print(case, nsteps, {k: f"{v:.2e}" for k, v in e.items()})
    bad = {k: v for k, v in e.items() if not v <= MIXED_TOL}
    assert not bad, bad


def test_mixed_tracers(dcm, orc):
    c = cases.sheared_convection(ip=16, jp=12, kp=12, ntracers=3)
    got, ref, errs = _run(dcm, orc, c, 2)
    e = _errors(c, got, ref)
    for q in range(3):
        e[f"q{q}"] = relerr(got["q"][q], ref["q"][q])
    print("tracers", {k: f"{v:.2e}" for k, v in e.items()})
    bad = {k: v for k, v in e.items() if not v <= MIXED_TOL}
    assert not bad, bad


@pytest.mark.parametrize("precision", [0, 1])
def test_graph_and_host_loops_agree(dcm, precision):
    """The graph-driven solve (conditional WHILE / IF nodes; with programmatic
    dependent launch and without) and the host-polled loop launch the same
    kernels in the same order: identical fields and iteration counts, step
    after step.  On a B200 the runtime takes programmatic launches inside the
    WHILE nodes, so mode 1 uses them."""
    c = small_bubble()
    out = []
    for mode in (1, 2, 0):
        core = dcm.DynamicalCore(c.grid)
        core.solver_graphs(mode)
        assert core.solver_graph_info()["programmatic_launch"] == (mode == 1)
        core.upload_state(c.state, c.dt, ptol=c.ptol, kord=c.kord, monotone=c.monotone,
                          precision=precision, precond=precision)
        core.driver_start()
        its = [core.step(1).iters_last for _ in range(3)]
        out.append((its, core.download_state()))
        core.close()
    ia, fa = out[0]
    for ib, fb in out[1:]:
        assert ia == ib
        for n in ("u", "v", "w", "th", "p", "psrc"):
            assert np.array_equal(fa[n], fb[n]), n


@pytest.mark.parametrize("fused", [1, 2])
@pytest.mark.parametrize("precond", [0, 1])
@pytest.mark.parametrize("shape", [(24, 20, 16), (9, 30, 37), (1, 16, 14), (40, 1, 12),
                                   (19, 37, 128)])
def test_fused_preconditioner_matches_unfused(dcm, shape, precond, fused):
    """The fused three-sweep preconditioner (FP32) performs each point's
    arithmetic of the three separate sweeps, unweighted and Chebyshev
    weighted, and with fused = 2 phase C's matvec t = A cs and its dots as a
    fourth stage: the launch shapes give the same iterations and fields to
    FP32 round-off, on strips and chunks that wrap (jp < 20, ip = 1), on
    ragged columns and on full 128-level columns."""
    ip, jp, kp = shape
    c = cases.warm_bubble(ip=ip, jp=jp, kp=kp, dxyz=50.0, radius=200.0, zc=200.0, seed=41)
    out = []
    for fuse in (fused, 0):
        core = dcm.DynamicalCore(c.grid)
        core.set_launch_shape(1, fuse=fuse)
        core.upload_state(c.state, c.dt, ptol=c.ptol, kord=c.kord, precision=1,
                          precond=precond)
        core.driver_start()
        its = [core.step(1).iters_last for _ in range(3)]
        out.append((its, core.download_state()))
        core.close()
    (ia, fa), (ib, fb) = out
    # the two launch shapes contract a few products into FMAs differently,
    # so the FP32 recursions part by round-off and stop a few iterations apart
    assert max(abs(a - b) for a, b in zip(ia, ib)) <= 4, (ia, ib)
    assert abs(sum(ia) - sum(ib)) <= 0.05 * sum(ib), (ia, ib)
    for n in ("u", "v", "w", "th"):
        assert relerr(fa[n], fb[n]) <= 1e-6, n


def test_chebyshev_sweeps_take_fewer_iterations(dcm):
    """The Chebyshev-weighted sweeps cost the same three operator
    applications as the reference's and converge in fewer FP32 iterations
    (the reference's preconditioned operator 1 - (1 - mu)^4 vanishes at the
    checkerboard modes' mu = 2 as well as at mu = 0)."""
    c = cases.warm_bubble(ip=48, jp=48, kp=32, dxyz=50.0, radius=500.0, zc=600.0, seed=43)
    its = {}
    for precond in (0, 1):
        core = dcm.DynamicalCore(c.grid)
        core.upload_state(c.state, c.dt, ptol=c.ptol, kord=c.kord, precision=1,
                          precond=precond)
        core.driver_start()
        st = [core.step(1) for _ in range(3)]
        assert all(s.err_last < c.ptol for s in st)
        its[precond] = sum(s.iters_last for s in st)
        core.close()
    print("FP32 iterations over 3 steps", its)
    assert its[1] < 0.85 * its[0], its


def test_mixed_solve_timeout_status(dcm):
    """The mixed form's graph-driven solve (a WHILE loop of FP64 update cycles
    around a WHILE loop of FP32 iterations) is bounded by the same round
    budget: a time step whose solve needs more rounds than the budget ends
    with DCM_E_TIMEOUT instead of hanging, and the handle runs normally once
    the default budget is back."""
    c = small_bubble()
    core = dcm.DynamicalCore(c.grid)
    try:
        def fresh():
            core.upload_state(c.state, c.dt, ptol=c.ptol, kord=c.kord, monotone=c.monotone,
                              precision=1, precond=1)
            core.driver_start()
        fresh()
        core.solver_limits(max_rounds=5)
        with pytest.raises(dcm.DCMError) as e:
            core.step(1)
        assert e.value.status == dcm.DCM_E_TIMEOUT
        core.solver_limits()
        fresh()
        st = core.step(1)
        assert st.err_last < c.ptol and st.iters_last > 5
    finally:
        core.close()


@pytest.mark.parametrize("shape", [(24, 20, 16), (9, 30, 37), (40, 1, 12), (12, 10, 70)])
def test_narrow_vectors_match_wide(dcm, shape):
    """The FP32 iteration kernels with 2 levels per lane (8-byte vectors,
    64-level warp tasks) against 4 levels per lane: the same operator, sweeps
    and dots, only the dot products' partition differs, so iterations and
    fields agree to FP32 round-off; columns of one, two and three warp tasks."""
    ip, jp, kp = shape
    c = cases.warm_bubble(ip=ip, jp=jp, kp=kp, dxyz=50.0, radius=200.0, zc=200.0, seed=44)
    out = []
    for vec in (2, 4):
        core = dcm.DynamicalCore(c.grid)
        core.set_launch_shape(1, fuse=0, vec=vec)
        core.upload_state(c.state, c.dt, ptol=c.ptol, kord=c.kord, precision=1, precond=1)
        core.driver_start()
        its = [core.step(1).iters_last for _ in range(3)]
        out.append((its, core.download_state()))
        core.close()
    (ia, fa), (ib, fb) = out
    assert max(abs(a - b) for a, b in zip(ia, ib)) <= 4, (ia, ib)
    for n in ("u", "v", "w", "th"):
        assert relerr(fa[n], fb[n]) <= 1e-6, n
