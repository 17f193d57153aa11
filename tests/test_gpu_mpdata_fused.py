"""The fused MPDATA iteration (one kernel per antidiffusive iteration:
antidiffusive velocities, the linked limiter and the first field's donor
cell, plane by plane in shared memory) against the separate per-stage
kernels, through the C-ABI.

Both evaluate the same point functions in the same order, so FP64 results
agree to round-off of FMA contraction (held at 1e-14 here; the oracle bar of
the drop-in tests is 1e-12).  Shapes cover ragged columns (k beyond one
warp), a single row (2-D x-z), several strips and chunks with wrapped halo
rows (a small row cap), and both limiter settings.
"""
import numpy as np
import pytest

from helpers import cases, rand_field, relerr, small_bubble, velocities

pytestmark = pytest.mark.gpu

SHAPES = [(24, 20, 16), (40, 1, 12), (17, 33, 70), (9, 7, 130)]


def _grid(shape):
    ip, jp, kp = shape
    if jp == 1:
        return cases.kelvin_helmholtz(ip=ip, jp=jp, kp=kp).grid
    return small_bubble(ip=ip, jp=jp, kp=kp).grid


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("kord,monotone", [(2, 1), (3, 1), (3, 0)])
@pytest.mark.parametrize("rows", [32, 5])
def test_fused_mpdata_3d_matches_separate_kernels(dcm, shape, kord, monotone, rows):
    g = _grid(shape)
    core = dcm.DynamicalCore(g)
    try:
        rng = np.random.default_rng(40 + kord)
        u, v, w = velocities(g, rng, 1.0, courant=0.2)
        psi = rand_field(g, rng, -0.3, 1.0)
        p_sep = psi.copy(order="F")
        p_fus = psi.copy(order="F")
        core.set_mpdata_shape(False)
        b_sep = core.mpdata_3d(1.0, u, v, w, p_sep, 0.1, -0.2, kord, monotone, 0, 0)
        core.set_mpdata_shape(True, rows)
        b_fus = core.mpdata_3d(1.0, u, v, w, p_fus, 0.1, -0.2, kord, monotone, 0, 0)
    finally:
        core.close()
    assert relerr(p_fus, p_sep) <= 1e-14
    assert b_fus == b_sep


@pytest.mark.parametrize("shape", SHAPES[:3])
def test_fused_mpdata_vec_3d_matches_separate_kernels(dcm, shape):
    g = _grid(shape)
    core = dcm.DynamicalCore(g)
    try:
        rng = np.random.default_rng(47)
        u, v, w = velocities(g, rng, 1.0, courant=0.2)
        fields = [rand_field(g, rng, -0.2, 1.0) for _ in range(3)]
        out = []
        for fuse in (False, True):
            q = dcm.fortran_stack(fields)
            lb, ub = np.array([0.0, 0.1, -0.1]), np.array([0.0, 0.2, 0.05])
            core.set_mpdata_shape(fuse, 7)
            core.mpdata_vec_3d(1.0, u, v, w, q, lb, ub, 3, 1, 0, 0)
            out.append((q, lb, ub))
    finally:
        core.close()
    (q0, lb0, ub0), (q1, lb1, ub1) = out
    for n in range(3):
        assert relerr(q1[n], q0[n]) <= 1e-14, n
    assert np.array_equal(lb0, lb1) and np.array_equal(ub0, ub1)


@pytest.mark.parametrize("precision", [0, 1])
def test_fused_mpdata_in_the_resident_step(dcm, precision):
    """Two resident time steps (theta's MPDATA with the source term added in
    the last donor-cell pass, and three passive tracers) with the fused and
    the separate MPDATA kernels: FP64 to round-off, FP32 within FP32
    round-off carried through a step."""
    c = cases.sheared_convection(ip=20, jp=18, kp=24, ntracers=3)
    res = []
    for fuse in (False, True):
        core = dcm.DynamicalCore(c.grid)
        try:
            core.set_mpdata_shape(fuse)
            core.upload_state(c.state, c.dt, ptol=c.ptol, kord=c.kord, monotone=c.monotone,
                              nq=c.nq, c_s=c.c_s, c_e=c.c_e, precision=precision)
            core.driver_start()
            core.step(2)
            res.append(core.download_state())
        finally:
            core.close()
    tol = 1e-12 if precision == 0 else 1e-5
    for n in ("u", "v", "w", "th"):
        assert relerr(res[1][n], res[0][n]) <= tol, n
    for q in range(3):
        assert relerr(res[1]["q"][q], res[0]["q"][q]) <= tol, q
