"""GPU parity of the Smagorinsky subgrid model (sgm/subgrid_3d.f90:38-493)
against the oracle, through the C-ABI: the stand-alone drop-in
(dcm_calculate_subgrid_3d, every inout field), exchange_full_wo, and the
resident time step with viscous = .true. in sources (dynamics.f90:878-893),
FP64 and mixed precision.

Bars as for the other routines: copies and exchanges bit-exact, the drop-in
1e-12 relative max-norm per field, the FP64 time step 1e-10 after one step
and 1e-8 after several, the mixed form 1e-5.
"""
import numpy as np
import pytest

from helpers import cases, fz, live_mask_p, rand_field, relerr, small_bubble, subgrid_inputs

pytestmark = pytest.mark.gpu

TOL = 1e-12
Z0 = 0.1  # roughness lengths of the reference's sgm/namelist.in
INOUT = ("vism", "vist", "strain", "tau11", "tau22", "tau33", "tau12", "tau13", "tau23",
         "su", "sv", "sw", "sth")


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


def test_exchange_full_wo(setup):
    g, core, ocore = setup
    rng = np.random.default_rng(40)
    a = rand_field(g, rng)
    b = a.copy(order="F")
    core.exchange_full_wo(a)
    ocore.exchange_full_wo(b)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("moisture", [False, True])
def test_calculate_subgrid_3d(setup, orc, moisture):
    g, core, ocore = setup
    lamsq = cases.mixing_length_sq(g, 0.23, Z0)
    a = subgrid_inputs(g, 41)
    b = {n: x.copy(order="F") for n, x in a.items()}
    kw_a, kw_b = {}, {}
    if moisture:
        rng = np.random.default_rng(42)
        qs = [rand_field(g, rng, 0.0, 1e-2) for _ in range(3)]
        sqs = [rand_field(g, rng, -1e-5, 1e-5) for _ in range(3)]
        for kw in (kw_a, kw_b):
            kw["q"] = orc._fortran_stack(qs)
            kw["sq"] = orc._fortran_stack(sqs)
            kw["viss"] = orc._fortran_stack([rand_field(g, rng) for _ in range(3)])
    names = ("u", "v", "w", "zu", "zv", "zw", "th") + INOUT
    core.calculate_subgrid_3d(lamsq, Z0, Z0, *[a[n] for n in names], **kw_a)
    ocore.calculate_subgrid_3d(lamsq, Z0, Z0, *[b[n] for n in names], **kw_b)
    errs = {n: relerr(a[n], b[n]) for n in INOUT}
    if moisture:
        for m in range(3):
            errs[f"sq{m}"] = relerr(kw_a["sq"][m], kw_b["sq"][m])
            assert np.array_equal(kw_a["viss"][m], a["vist"])
    bad = {k: v for k, v in errs.items() if not v <= TOL}
    assert not bad, bad
    # inputs untouched, the viscosities live
    for n in ("u", "v", "w", "zu", "zv", "zw", "th"):
        assert np.array_equal(a[n], b[n])
    assert np.max(a["vism"][1:g.kp - 1]) > 0.0


def _viscous(g):
    return dict(lamsq=cases.mixing_length_sq(g, 0.23, Z0), z0=Z0, z0th=Z0)


def _run(dcm, orc, c, nsteps, precision=0):
    vis = _viscous(c.grid)
    core = dcm.DynamicalCore(c.grid)
    core.upload_state(c.state, c.dt, ptol=c.ptol, kord=c.kord, monotone=c.monotone, nq=c.nq,
                      c_s=c.c_s, c_e=c.c_e, precision=precision, viscous=vis)
    core.driver_start()
    its = [core.step(1).iters_last for _ in range(nsteps)]
    got = core.download_state()
    core.close()
    m = orc.OracleModel(c.grid, c.state, c.dt, ptol=c.ptol, kord=c.kord, monotone=c.monotone,
                        nq=c.nq, c_s=c.c_s, c_e=c.c_e, viscous=vis)
    m.driver_start()
    oits = [m.step(1)[0] for _ in range(nsteps)]
    return got, m.fields(), its, oits


def _errors(c, got, ref, names):
    e = {n: relerr(got[n], ref[n]) for n in names}
    e["p"] = relerr(got["p"], ref["p"], live_mask_p(c.grid))
    return e


STEP_FIELDS = ("u", "v", "w", "zu", "zv", "zw", "th", "su", "sv", "sw", "sth")


@pytest.mark.parametrize("nsteps,tol", [(1, 1e-10), (4, 1e-8)])
def test_viscous_step(dcm, orc, nsteps, tol):
    c = small_bubble()
    got, ref, its, oits = _run(dcm, orc, c, nsteps)
    assert max(abs(a - b) for a, b in zip(its, oits)) <= 1
    e = _errors(c, got, ref, STEP_FIELDS)
    print("viscous", nsteps, {k: f"{v:.2e}" for k, v in e.items()})
    bad = {k: v for k, v in e.items() if not v <= tol}
    assert not bad, bad
    # the subgrid terms are live: the step differs from the inviscid one
    core = dcm.DynamicalCore(c.grid)
    core.upload_state(c.state, c.dt, ptol=c.ptol, kord=c.kord, monotone=c.monotone)
    core.driver_start()
    core.step(nsteps)
    inv = core.download_state()
    core.close()
    assert relerr(inv["th"], got["th"]) > 1e-8


def test_viscous_step_tracers(dcm, orc):
    c = cases.sheared_convection(ip=16, jp=12, kp=12, ntracers=3)
    got, ref, its, oits = _run(dcm, orc, c, 2)
    e = _errors(c, got, ref, STEP_FIELDS)
    for q in range(3):
        e[f"q{q}"] = relerr(got["q"][q], ref["q"][q])
    bad = {k: v for k, v in e.items() if not v <= 1e-10}
    assert not bad, bad


def test_viscous_step_mixed(dcm, orc):
    c = small_bubble()
    got, ref, _, _ = _run(dcm, orc, c, 3, precision=1)
    e = _errors(c, got, ref, ("u", "v", "w", "th"))
    print("viscous mixed", {k: f"{v:.2e}" for k, v in e.items()})
    bad = {k: v for k, v in e.items() if not v <= 1e-5}
    assert not bad, bad
