"""GPU parity of the PAMM sedimentation transport (dcm_mpdata_vec_1d:
mpdata_vec_1d, pamm/sfvt/advection_1d.F90:463-778, batched over columns with
the caller's sub-steps, pamm/microphysics.f90:3139-3183) against the oracle,
through the C-ABI.

FP64 on both sides; the GPU contracts products into FMAs, so the bar is
1e-12 relative max-norm per column and field (the drop-ins' bar).  Cases:
every combination of the scheme's options, columns taller than one warp's
32 levels (each lane then owns several), several halo widths, per-column
metrics and sub-step counts, an all-zero column (the early return), and the
sedimentation form the microphysics calls (kord 1, fall speeds from the
column's largest Courant number).
"""
import numpy as np
import pytest

from helpers import relerr
from test_oracle_column import _columns

pytestmark = pytest.mark.gpu


def _check(dcm, orc, met, w, psi, dt, nsub, **kw):
    a = psi.copy()
    b = psi.copy()
    dcm.mpdata_vec_1d_columns(dt, nsub, *met, w, a, **kw)
    orc.mpdata_vec_1d_columns(dt, nsub, *met, w, b, **kw)
    assert np.all(np.isfinite(a))
    for c in range(psi.shape[0]):
        for n in range(psi.shape[1]):
            assert relerr(a[c, n], b[c, n]) <= 1e-12, (c, n)
    return a


@pytest.mark.parametrize("kord,monotone", [(1, 0), (2, 0), (2, 1), (3, 1), (3, 0)])
@pytest.mark.parametrize("neumann", [0, 1, 2])
@pytest.mark.parametrize("kp", [23, 130])
def test_column_transport_matches_the_oracle(dcm, orc, kord, monotone, neumann, kp):
    ncol, nq = 9, 3
    met, w, psi = _columns(100 + kord + 3 * monotone + 7 * neumann + kp, ncol, nq, kp, 1, 1,
                           False, zero_col=True)
    dt = np.linspace(0.5, 2.0, ncol)
    nsub = (1 + np.arange(ncol) % 3).astype(np.int32)
    out = _check(dcm, orc, met, w, psi, dt, nsub, kord=kord, monotone=monotone,
                 neumann=neumann)
    assert np.array_equal(out[0], psi[0])  # all zero: unchanged


@pytest.mark.parametrize("l_h,r_h", [(2, 2), (1, 3), (3, 1)])
def test_column_transport_halo_widths_per_column_metrics(dcm, orc, l_h, r_h):
    ncol, nq, kp = 37, 2, 61
    met, w, psi = _columns(200 + l_h + 5 * r_h, ncol, nq, kp, l_h, r_h, True)
    _check(dcm, orc, met, w, psi, 1.0, 2, kord=3, monotone=True, l_h=l_h, r_h=r_h)


def test_sedimentation_form_many_columns(dcm, orc):
    """The calls of the microphysics: kord 1, no limiter, fall speeds at the
    faces, n_step = max(ceiling(max |v| dt / dz * 2), 1) per column."""
    ncol, nq, kp = 513, 2, 120
    met, w, psi = _columns(300, ncol, nq, kp, 1, 1, False, fall=8.0)
    dt = 2.0
    nsub = np.maximum(np.ceil(np.max(np.abs(w), axis=1) * dt / met[0].min() * 2.0), 1)
    _check(dcm, orc, met, w, psi, dt, nsub.astype(np.int32), kord=1)


def test_column_transport_rejects_bad_arguments(dcm):
    met, w, psi = _columns(5, 2, 1, 10, 1, 1, False)
    with pytest.raises(dcm.DCMError):
        dcm.mpdata_vec_1d_columns(1.0, [1, 0], *met, w, psi.copy())  # nsub < 1
    lib = dcm.library()
    assert lib.dcm_mpdata_vec_1d(2, 10, 1, 0, 1, None, None, None, None, None, None, 0, None,
                                 None, 1, 0, 0) == dcm.DCM_E_ARG  # l_h < 1


def test_device_entry_point_matches_the_host_one(dcm):
    """dcm_mpdata_vec_1d_device on device arrays, queued on a stream, gives
    the host entry point's result bit for bit (the same kernel)."""
    import ctypes as C

    import torch

    ncol, nq, kp = 70, 3, 45
    met, w, psi = _columns(400, ncol, nq, kp, 1, 1, True)
    dt = np.linspace(0.5, 2.0, ncol)
    nsub = (1 + np.arange(ncol) % 4).astype(np.int32)
    ref = psi.copy()
    dcm.mpdata_vec_1d_columns(dt, nsub, *met, w, ref, kord=3, monotone=True, neumann=1)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to("cuda")  # noqa: E731
    d_dt, d_ns, d_w, d_psi = dev(dt), dev(nsub), dev(w), dev(psi)
    d_met = [dev(a) for a in met]
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()  # the uploads (on torch's stream) have landed
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    st = dcm.library().dcm_mpdata_vec_1d_device(
        ncol, kp, nq, 1, 1, p(d_dt), p(d_ns), *[p(t) for t in d_met], kp + 2, p(d_w), p(d_psi),
        3, 1, 1, C.c_void_p(stream.cuda_stream))
    assert st == dcm.DCM_OK
    stream.synchronize()
    assert np.array_equal(d_psi.cpu().numpy(), ref)
