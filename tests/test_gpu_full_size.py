"""GPU checks at the benchmark's full size, the 256x256x128 warm bubble, through
properties that hold at any size (the oracle's CPU step at this size takes
too long for a test; its parity is tested on the smaller grids):

* every pressure solve converges to ptol on its FP64 residual, in both forms;
* the mixed form stays within the mixed-precision configuration's bars of
  the FP64 path (p <= 1e-6 relative max-norm with the mean removed, on its
  live cells; velocities <= 1e-5), the comparison the benchmark reports;
* the graph-driven and the host-polled solver loops give bit-identical
  fields (deterministic reductions, the same kernels in the same order).
"""
import numpy as np
import pytest

from helpers import cases, live_mask_p, relerr

pytestmark = pytest.mark.gpu

STEPS = 2


@pytest.fixture(scope="module")
def bubble():
    return cases.warm_bubble()


def _run(dcm, c, precision, graphs=1):
    core = dcm.DynamicalCore(c.grid)
    core.solver_graphs(graphs)
    core.upload_state(c.state, c.dt, ptol=c.ptol, kord=c.kord, monotone=c.monotone,
                      precision=precision, precond=precision)
    core.driver_start()
    stats = [core.step(1) for _ in range(STEPS)]
    out = core.download_state()
    core.close()
    return stats, out


def test_mixed_form_within_its_bars_of_the_fp64_path(dcm, bubble):
    g = bubble.grid
    assert (g.ip, g.jp, g.kp) == (256, 256, 128)
    s64, f64 = _run(dcm, bubble, 0)
    s32, f32 = _run(dcm, bubble, 1)
    for s in s64 + s32:
        assert s.iters_last > 0 and s.err_last < bubble.ptol
    m = live_mask_p(g)
    p32, p64 = f32["p"][m], f64["p"][m]
    assert relerr(p32 - p32.mean(), p64 - p64.mean()) <= 1e-6
    for n in ("u", "v", "w"):
        assert relerr(f32[n], f64[n]) <= 1e-5, n
    assert relerr(f32["th"], f64["th"]) <= 1e-5


def test_graph_and_host_loops_agree_at_full_size(dcm, bubble):
    sa, fa = _run(dcm, bubble, 1, graphs=1)
    sb, fb = _run(dcm, bubble, 1, graphs=0)
    assert [s.iters_last for s in sa] == [s.iters_last for s in sb]
    for n in ("u", "v", "w", "th", "p"):
        assert np.array_equal(fa[n], fb[n]), n


def test_sheared_convection_mixed_form_against_the_fp64_path(dcm):
    """The 512x512x256 sheared convection with 8 FP32 tracers (the scale
    configuration), steps 1..10 in both forms: every pressure solve converges
    to ptol on its FP64 residual, and the mixed form stays within the bars
    this turbulent case holds it to against the FP64 path.  The bars are the
    measured differences after 10 steps (v 2.4e-6, p 8.5e-6) with a margin of
    about 3x: FP32 round-off seeds differences that the shear-driven
    convection amplifies step by step, so this case's p difference is above
    the warm bubble's 1e-6 bar, which that configuration states for its own,
    smoother case."""
    c = cases.sheared_convection()
    g = c.grid
    assert (g.ip, g.jp, g.kp) == (512, 512, 256) and c.nq == 8
    out = []
    for precision in (0, 1):
        core = dcm.DynamicalCore(g)
        core.upload_state(c.state, c.dt, ptol=c.ptol, kord=c.kord, monotone=c.monotone,
                          nq=c.nq, c_s=c.c_s, c_e=c.c_e, precision=precision,
                          precond=precision)
        core.driver_start()
        stats = [core.step(1) for _ in range(10)]
        for s in stats:
            assert s.iters_last > 0 and s.err_last < c.ptol
        f = core.download_state()
        out.append({k: np.array(f[k], copy=True) for k in ("u", "v", "w", "th", "p")} |
                   {"q": [np.array(q, copy=True) for q in f["q"]]})
        core.close()
    f64, f32 = out
    m = live_mask_p(g)
    p32, p64 = f32["p"][m], f64["p"][m]
    assert relerr(p32 - p32.mean(), p64 - p64.mean()) <= 3e-5
    for n in ("u", "v", "w", "th"):
        assert relerr(f32[n], f64[n]) <= 1e-5, n
    for q in range(c.nq):
        assert relerr(f32["q"][q], f64["q"][q]) <= 1e-4, q
