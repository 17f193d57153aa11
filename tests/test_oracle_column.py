"""CPU tests of the oracle's PAMM sedimentation transport (mpdata_vec_1d,
pamm/sfvt/advection_1d.F90:463-778, with the caller's sub-steps): bit for bit
against the independent numpy restatement (tests/column_np.py) over the
scheme's options, halo widths, per-column metrics and sub-step counts, and
the all-zero early return."""
import numpy as np
import pytest

import column_np
from conftest import load_oracle


def _columns(seed, ncol, nq, kp, l_h, r_h, per_column, fall=3.0, zero_col=False):
    rng = np.random.default_rng(seed)
    nw, npsi = kp + l_h + r_h, kp + 2 * r_h
    z = np.linspace(0.0, 1.0, nw)
    shape = (ncol, nw) if per_column else (nw,)
    dz = np.broadcast_to(40.0 + 20.0 * z, shape) * (1.0 + 0.1 * rng.random(shape))
    dzn = np.broadcast_to(45.0 + 10.0 * z, shape) * (1.0 + 0.1 * rng.random(shape))
    rhoa = np.broadcast_to(1.2 - 0.5 * z, shape) * (1.0 + 0.05 * rng.random(shape))
    rhoan = np.broadcast_to(1.2 - 0.5 * z, shape) * (1.0 + 0.05 * rng.random(shape))
    # fall speeds as the microphysics passes them: negative (downward) at the
    # faces, a column-dependent magnitude
    w = -fall * rng.random((ncol, nw)) * rng.random((ncol, 1))
    psi = rng.random((ncol, nq, npsi)) * (rng.random((ncol, nq, npsi)) > 0.3)
    psi[:, :, :] *= 1e-3
    if zero_col:
        psi[0] = 0.0
    return [np.ascontiguousarray(a) for a in (dz, dzn, rhoa, rhoan)], w, psi


@pytest.mark.parametrize("kord,monotone", [(1, 0), (2, 0), (2, 1), (3, 1), (3, 0)])
@pytest.mark.parametrize("neumann", [0, 1, 2])
def test_column_transport_matches_numpy(kord, monotone, neumann):
    orc = load_oracle()
    ncol, nq, kp = 5, 3, 23
    met, w, psi = _columns(10 + kord + 3 * monotone + 7 * neumann, ncol, nq, kp, 1, 1, False,
                           zero_col=True)
    dt = np.array([2.0, 1.0, 0.5, 2.0, 1.5])
    nsub = np.array([1, 2, 3, 1, 4], dtype=np.int32)
    a = psi.copy()
    b = psi.copy()
    orc.mpdata_vec_1d_columns(dt, nsub, *met, w, a, kord=kord, monotone=monotone,
                              neumann=neumann)
    column_np.columns(dt, nsub, *met, w, b, kord=kord, monotone=monotone, neumann=neumann)
    assert np.array_equal(a, b)
    assert not np.array_equal(a[1:], psi[1:])   # the columns moved
    assert np.array_equal(a[0], psi[0])         # all zero: returned unchanged


@pytest.mark.parametrize("l_h,r_h", [(2, 2), (1, 3), (3, 1)])
def test_column_transport_halo_widths_and_metrics_per_column(l_h, r_h):
    orc = load_oracle()
    ncol, nq, kp = 4, 2, 17
    met, w, psi = _columns(30 + l_h + 5 * r_h, ncol, nq, kp, l_h, r_h, True)
    a = psi.copy()
    b = psi.copy()
    orc.mpdata_vec_1d_columns(1.0, 2, *met, w, a, kord=3, monotone=True, l_h=l_h, r_h=r_h)
    column_np.columns(1.0, 2, *met, w, b, kord=3, monotone=True, l_h=l_h, r_h=r_h)
    assert np.array_equal(a, b)


def test_donor_cell_sedimentation_keeps_fields_non_negative():
    """kord 1 (the sedimentation calls, pamm/microphysics.f90:3141-3183) at
    a Courant number below one per sub-step keeps every field non-negative
    and, with empty halos, only loses density-weighted mass (through the
    bottom face): sum(rhoan dzn psi) telescopes to the boundary fluxes."""
    orc = load_oracle()
    ncol, nq, kp = 6, 2, 40
    met, w, psi = _columns(77, ncol, nq, kp, 1, 1, False, fall=5.0)
    psi[:, :, 0] = 0.0
    psi[:, :, -1] = 0.0
    dz, dzn, _, rhoan = met
    nsub = np.maximum(np.ceil(np.max(np.abs(w), axis=1) * 2.0 / dz.min() * 2.0), 1)
    a = psi.copy()
    orc.mpdata_vec_1d_columns(2.0, nsub.astype(np.int32), *met, w, a, kord=1)
    assert np.all(a[:, :, 1:-1] >= 0.0)
    mass = lambda x: (x[:, :, 1:-1] * (rhoan * dzn)[1:-1]).sum(axis=2)  # noqa: E731
    assert np.all(mass(a) <= mass(psi) * (1 + 1e-14))
    assert np.any(mass(a) < mass(psi) * (1 - 1e-6))
