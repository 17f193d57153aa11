"""GPU checks of the batched ensemble (one CUDA graph launch per time step
for all members) and of the solver launch-shape autotuner.

An ensemble member runs exactly the kernels a standalone handle runs for
the same state, in the same order, with per-member reductions of fixed
order, so its fields must be bit-identical to the standalone run; each
member's pressure solve stops at its own convergence (per-member masks).
"""
import numpy as np
import pytest

from helpers import cases, relerr, small_bubble

pytestmark = pytest.mark.gpu

SIZES = [(24, 20, 16, 2.0), (16, 24, 12, 1.0), (32, 16, 20, 3.0)]


def _members():
    return [cases.warm_bubble(ip=ip, jp=jp, kp=kp, dxyz=50.0, amp=amp, radius=300.0, zc=400.0,
                              seed=10 + n) for n, (ip, jp, kp, amp) in enumerate(SIZES)]


def _upload(core, c, precision, **kw):
    core.upload_state(c.state, c.dt, ptol=c.ptol, kord=c.kord, monotone=c.monotone,
                      precision=precision, **kw)
    core.driver_start()


def _options(c, opts):
    kw = {}
    if "cheb" in opts:
        kw.update(precond=1, precond_lo=0.05)
    if "viscous" in opts:
        kw["viscous"] = dict(lamsq=cases.mixing_length_sq(c.grid, 0.23, 0.1), z0=0.1, z0th=0.1)
    return kw


@pytest.mark.parametrize("precision,opts", [(0, ()), (1, ()), (1, ("cheb",)),
                                            (0, ("viscous",)), (1, ("cheb", "viscous"))])
def test_ensemble_matches_standalone(dcm, precision, opts):
    """Also with the Chebyshev-weighted sweeps and with the subgrid model in
    the captured step."""
    cs = _members()
    ens = dcm.Ensemble([c.grid for c in cs])
    for core, c in zip(ens.members, cs):
        _upload(core, c, precision, **_options(c, opts))
    its_e = []
    for _ in range(4):
        st = ens.step(1)
        assert st.steps == 1
        its_e.append([m.last_iters() for m in ens.members])
    got = [m.download_state() for m in ens.members]
    ens.close()
    for n, c in enumerate(cs):
        core = dcm.DynamicalCore(c.grid)
        _upload(core, c, precision, **_options(c, opts))
        its = [core.step(1).iters_last for _ in range(4)]
        ref = core.download_state()
        core.close()
        assert its == [row[n] for row in its_e]
        for f in ("u", "v", "w", "th", "p"):
            assert np.array_equal(got[n][f], ref[f]), (n, f)
    # members of different sizes and amplitudes converge after different
    # numbers of iterations within the same graph launch
    assert len({tuple(r) for r in zip(*its_e)}) > 1


def test_ensemble_rejects_members_at_different_steps(dcm):
    cs = _members()[:2]
    ens = dcm.Ensemble([c.grid for c in cs])
    for core, c in zip(ens.members, cs):
        _upload(core, c, 1)
    ens.members[0].step(1)
    with pytest.raises(dcm.DCMError) as e:
        ens.step(1)
    assert e.value.status == dcm.DCM_E_ARG
    ens.close()


def test_tune_and_cache(dcm, tmp_path, monkeypatch):
    monkeypatch.setenv("DCM_TUNE_CACHE", str(tmp_path / "tune.txt"))
    c = small_bubble()
    core = dcm.DynamicalCore(c.grid)
    by, tasks, depth, fuse, vec = core.tune(precision=1, use_cache=True)
    assert by in (2, 4, 8) and tasks in (0, 1, 2) and depth in (1, 2, 4, 8)
    assert fuse in (0, 1, 2) and vec in (2, 4) and not (fuse and vec != 4)
    lines = (tmp_path / "tune.txt").read_text().splitlines()
    assert len(lines) == 1
    # from the cache
    assert core.tune(precision=1, use_cache=True) == (by, tasks, depth, fuse, vec)
    assert len((tmp_path / "tune.txt").read_text().splitlines()) == 1
    # the tuned shape changes only the order of the dot-product sums
    _upload(core, c, 0)
    core.step(2)
    a = core.download_state()
    core.close()
    ref = dcm.DynamicalCore(c.grid)
    _upload(ref, c, 0)
    ref.step(2)
    b = ref.download_state()
    ref.close()
    for f in ("u", "v", "w", "th"):
        assert relerr(a[f], b[f]) <= 1e-8, f
