"""GPU parity of the device-resident time loop (model_driver's dry step)
against the oracle's restatement of the same loop.

Bar: 1e-10 relative max-norm per field after one step (the FP64 parity bar).
After several steps the two runs drift apart only through round-off of the
iterative solve (tolerance 1e-10 on the residual); the multi-step tolerance
is 1e-8 per field.
"""
import numpy as np
import pytest

from helpers import cases, live_mask_p, relerr, small_bubble

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "w", "zu", "zv", "zw", "th", "su", "sv", "sw", "psrc", "div", "sth")


def _run(dcm, orc, c, nsteps, **kw):
    core = dcm.DynamicalCore(c.grid)
    core.upload_state(c.state, c.dt, ptol=c.ptol, kord=c.kord, monotone=c.monotone,
                      nq=c.nq, c_s=c.c_s, c_e=c.c_e, **kw)
    core.driver_start()
    its = [core.step(1).iters_last for _ in range(nsteps)]
    got = core.download_state()
    core.close()
    okw = {k: v for k, v in kw.items() if k != "precision"}  # the oracle is FP64
    m = orc.OracleModel(c.grid, c.state, c.dt, ptol=c.ptol, kord=c.kord, monotone=c.monotone,
                        nq=c.nq, c_s=c.c_s, c_e=c.c_e, **okw)
    m.driver_start()
    oits = [m.step(1)[0] for _ in range(nsteps)]
    return got, m.fields(), its, oits


def _scaled(a, b, scale):
    """max|a - b| relative to max(max|b|, scale): quantities that are zero up
    to round-off (the projected divergence, the level means of v and w) are
    measured against the size of the terms they are made of."""
    num = np.max(np.abs(np.asarray(a) - np.asarray(b)))
    den = max(np.max(np.abs(b)), scale)
    return num / den if den > 0 else num


def _compare(c, got, ref, tol):
    g = c.grid
    errs = {}
    for n in FIELDS:
        errs[n] = relerr(got[n], ref[n])
    # div = sum of three rho*du/dx terms that cancel to round-off
    vmax = max(np.max(np.abs(ref[n])) for n in ("u", "v", "w"))
    errs["div"] = _scaled(got["div"], ref["div"], np.max(g.rhoa) * vmax / g.dz[1])
    errs["p"] = relerr(got["p"], ref["p"], live_mask_p(g))
    for n, fld in (("ubar", "u"), ("vbar", "v"), ("wbar", "w"), ("thbar", "th")):
        errs[n] = _scaled(got[n], ref[n], np.max(np.abs(ref[fld])))
    bad = {k: v for k, v in errs.items() if not v <= tol}
    assert not bad, bad
    return errs


@pytest.mark.parametrize("case", ["bubble", "kh"])
def test_one_step(dcm, orc, case):
    c = small_bubble() if case == "bubble" else cases.kelvin_helmholtz(ip=40, jp=1, kp=12)
    got, ref, its, oits = _run(dcm, orc, c, 1)
    assert its == oits
    _compare(c, got, ref, 1e-10)


def test_ten_steps_bubble(dcm, orc):
    c = small_bubble()
    got, ref, its, oits = _run(dcm, orc, c, 10)
    assert max(abs(a - b) for a, b in zip(its, oits)) <= 1
    _compare(c, got, ref, 1e-8)


@pytest.mark.parametrize("scheme,limiter", [(0, 0), (2, 0), (1, 1)])
def test_scheme_variants(dcm, orc, scheme, limiter):
    c = small_bubble(ip=16, jp=12, kp=12)
    kw = dict(advection_scheme=scheme, limiter=limiter)
    if scheme == 2:
        kw.update(thbase=float(c.grid.thetan[0]), thtop=float(c.grid.thetan[-1]))
    got, ref, its, oits = _run(dcm, orc, c, 2, **kw)
    _compare(c, got, ref, 1e-10)


def test_tracers(dcm, orc):
    c = cases.sheared_convection(ip=16, jp=12, kp=12, ntracers=3)
    got, ref, its, oits = _run(dcm, orc, c, 2)
    _compare(c, got, ref, 1e-10)
    for q in range(3):
        assert relerr(got["q"][q], ref["q"][q]) <= 1e-10


def test_damping_forcing(dcm, orc):
    c = small_bubble(ip=16, jp=12, kp=12)
    K2 = c.grid.kp + 2
    z = c.grid.z
    forcing = dict(damping_layer=1, forcing=1, divergence=1,
                   dampfacn=np.where(c.grid.zn > 800.0, -1.0 / 300.0, 0.0),
                   dampfac=np.where(z > 800.0, -1.0 / 300.0, 0.0),
                   u_force=np.full(K2, 0.5), v_force=np.full(K2, -0.25),
                   w_subs=-1e-5 * z, forcing_tau=900.0)
    got, ref, its, oits = _run(dcm, orc, c, 2, forcing=forcing)
    _compare(c, got, ref, 1e-10)


@pytest.mark.parametrize("shape", [(12, 10, 13), (8, 6, 130), (1, 16, 14), (10, 1, 9)])
def test_ragged_and_degenerate_shapes(dcm, orc, shape):
    """Column heights that are not a multiple of the 16-byte vector (13, 9),
    columns longer than one warp's vector span (130 levels: two k-chunks in
    both precisions), and the 2-D forms of the reference (ip = 1: y-z,
    jp = 1: x-z) against the oracle after two steps."""
    ip, jp, kp = shape
    c = cases.warm_bubble(ip=ip, jp=jp, kp=kp, dxyz=50.0, radius=200.0, zc=200.0, seed=31)
    # solved to 1e-13 so that a stopping point one iteration apart (dot
    # products summed in another order) leaves round-off, not tolerance-sized,
    # differences: any error at the vector or k-chunk seams would stand out
    c.ptol = 1e-13
    got, ref, its, oits = _run(dcm, orc, c, 2)
    # near the round-off floor the stopping iteration varies by a few
    assert max(abs(a - b) for a, b in zip(its, oits)) <= 3
    errs = _compare(c, got, ref, 1e-10)
    assert errs["p"] <= 1e-10


@pytest.mark.parametrize("shape", [(12, 10, 13), (8, 6, 130), (1, 16, 14)])
def test_ragged_shapes_mixed(dcm, orc, shape):
    ip, jp, kp = shape
    c = cases.warm_bubble(ip=ip, jp=jp, kp=kp, dxyz=50.0, radius=200.0, zc=200.0, seed=32)
    got, ref, _, _ = _run(dcm, orc, c, 2, precision=1)
    for n in ("u", "v", "w", "th"):
        assert relerr(got[n], ref[n]) <= 1e-5, n
    assert relerr(got["p"], ref["p"], live_mask_p(c.grid)) <= 1e-5


@pytest.mark.parametrize("precision", [0, 1])
def test_reupload_with_the_same_layout(dcm, precision):
    """A second dcm_state_upload of the same layout keeps the device buffers
    (zeroed) and the captured solves: the steps that follow are bit-identical
    to those of a fresh handle, after a first run that left every buffer
    dirty; a layout change (moisture on) still works."""
    c1 = cases.sheared_convection(ip=16, jp=12, kp=12, ntracers=2, seed=5)
    c2 = cases.sheared_convection(ip=16, jp=12, kp=12, ntracers=2, seed=6)
    kw = dict(nq=2, c_s=c1.c_s, c_e=c1.c_e, precision=precision)
    core = dcm.DynamicalCore(c1.grid)
    core.upload_state(c1.state, c1.dt, ptol=c1.ptol, kord=c1.kord, **kw)
    core.driver_start()
    core.step(3)
    core.upload_state(c2.state, c2.dt, ptol=c2.ptol, kord=c2.kord, **kw)
    core.driver_start()
    its = [core.step(1).iters_last for _ in range(3)]
    got = core.download_state()
    fresh = dcm.DynamicalCore(c2.grid)
    fresh.upload_state(c2.state, c2.dt, ptol=c2.ptol, kord=c2.kord, **kw)
    fresh.driver_start()
    its_f = [fresh.step(1).iters_last for _ in range(3)]
    ref = fresh.download_state()
    fresh.close()
    assert its == its_f
    for n in ("u", "v", "w", "th", "p", "su", "sth", "psrc", "div"):
        assert np.array_equal(got[n], ref[n]), n
    for q in range(2):
        assert np.array_equal(got["q"][q], ref["q"][q]), q
    # another layout on the same handle: no tracers
    core.upload_state(c2.state, c2.dt, ptol=c2.ptol, kord=c2.kord, precision=precision)
    core.driver_start()
    assert core.step(2).err_last < c2.ptol
    core.close()


def test_small_solver_in_the_resident_step(dcm, orc):
    """The 2-D shear layer's resident FP64 step with the one-cluster solve
    (the default at this size) and with the multi-kernel solve: the same
    fields to the solve's tolerance; the iteration counts part by summation-
    order round-off (a few per step, as the reference's own counts do under a
    change of decomposition), so they are held within 5 per step and 5 % in
    total."""
    c = cases.kelvin_helmholtz(ip=64, jp=1, kp=32)
    out = []
    for small in (8192, 0):
        core = dcm.DynamicalCore(c.grid)
        core.set_small_solver(small)
        core.upload_state(c.state, c.dt, ptol=c.ptol, kord=c.kord, monotone=c.monotone)
        core.driver_start()
        its = [core.step(1).iters_last for _ in range(5)]
        out.append((its, core.download_state()))
        core.close()
    (ia, fa), (ib, fb) = out
    assert max(abs(x - y) for x, y in zip(ia, ib)) <= 5, (ia, ib)
    assert abs(sum(ia) - sum(ib)) <= 0.05 * sum(ib), (ia, ib)
    for n in ("u", "w", "th"):
        assert relerr(fa[n], fb[n]) <= 1e-8, n
