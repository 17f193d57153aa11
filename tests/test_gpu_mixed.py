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


def _run(dcm, orc, c, nsteps, **kw):
    core = dcm.DynamicalCore(c.grid)
    core.upload_state(c.state, c.dt, ptol=c.ptol, kord=c.kord, monotone=c.monotone,
                      nq=c.nq, c_s=c.c_s, c_e=c.c_e, precision=1, **kw)
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


@pytest.mark.parametrize("case,nsteps", [("bubble", 1), ("kh", 1), ("bubble", 10)])
def test_mixed_against_oracle(dcm, orc, case, nsteps):
    c = small_bubble() if case == "bubble" else cases.kelvin_helmholtz(ip=40, jp=1, kp=12)
    got, ref, errs = _run(dcm, orc, c, nsteps)
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
    """The graph-driven solve (conditional WHILE / IF nodes) and the
    host-polled loop launch the same kernels in the same order: identical
    fields and iteration counts, step after step."""
    c = small_bubble()
    out = []
    for graphs in (True, False):
        core = dcm.DynamicalCore(c.grid)
        core.solver_graphs(graphs)
        core.upload_state(c.state, c.dt, ptol=c.ptol, kord=c.kord, monotone=c.monotone,
                          precision=precision)
        core.driver_start()
        its = [core.step(1).iters_last for _ in range(3)]
        out.append((its, core.download_state()))
        core.close()
    (ia, fa), (ib, fb) = out
    assert ia == ib
    for n in ("u", "v", "w", "th", "p", "psrc"):
        assert np.array_equal(fa[n], fb[n]), n


@pytest.mark.parametrize("shape", [(24, 20, 16), (9, 30, 37), (1, 16, 14), (40, 1, 12)])
def test_fused_preconditioner_matches_unfused(dcm, shape):
    """The fused three-sweep preconditioner (FP32) performs each point's
    arithmetic of the three separate sweeps: the two launch shapes give the
    same iterations and fields to FP32 round-off, on strips and chunks that
    wrap (jp < 20, ip = 1) and on ragged columns."""
    ip, jp, kp = shape
    c = cases.warm_bubble(ip=ip, jp=jp, kp=kp, dxyz=50.0, radius=200.0, zc=200.0, seed=41)
    out = []
    for fuse in (1, 0):
        core = dcm.DynamicalCore(c.grid)
        core.set_launch_shape(1, fuse=fuse)
        core.upload_state(c.state, c.dt, ptol=c.ptol, kord=c.kord, precision=1)
        core.driver_start()
        its = [core.step(1).iters_last for _ in range(3)]
        out.append((its, core.download_state()))
        core.close()
    (ia, fa), (ib, fb) = out
    assert max(abs(a - b) for a, b in zip(ia, ib)) <= 2
    for n in ("u", "v", "w", "th"):
        assert relerr(fa[n], fb[n]) <= 1e-6, n
