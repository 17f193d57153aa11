"""The allocation-free horizontal means (dcm_horizontal_means_noalloc).

For hosts that own all device memory through their own pool or budget and
do not let library code call cudaMalloc / cudaFree: the caller passes device
pointers and a stream, and the reduction uses a fixed scratch array inside
the library.  This file is collected last on purpose.  It checks, on two
calls in a row (the scratch is reused and must leave no state behind), that
the result equals the handle-based dcm_horizontal_means on the same fields.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import rand_field, relerr, small_bubble

pytestmark = pytest.mark.gpu


def test_means_without_allocation_match_the_handle_api(dcm):
    import torch

    g = small_bubble(ip=36, jp=28, kp=20, seed=11).grid
    rng = np.random.default_rng(77)
    fields = [rand_field(g, rng) for _ in range(4)]
    core = dcm.DynamicalCore(g)
    ref = core.horizontal_means(*fields)[:4]
    core.close()
    K2 = g.kp + 2
    expected = np.concatenate(ref)

    lib = dcm.library()
    dev = [torch.from_numpy(np.ravel(a, order="F").copy()).to("cuda") for a in fields]
    out = torch.empty(4 * K2, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    for call in range(2):
        out.fill_(float("nan"))
        st = lib.dcm_horizontal_means_noalloc(
            g.ip, g.jp, g.kp, *[C.c_void_p(t.data_ptr()) for t in dev],
            C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert st == dcm.DCM_OK, (call, st)
        stream.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got)), call
        assert relerr(got, expected) <= 1e-12, call


def test_means_without_allocation_reject_oversize_levels(dcm):
    lib = dcm.library()
    st = lib.dcm_horizontal_means_noalloc(8, 8, 1025, None, None, None, None, None, None)
    assert st == dcm.DCM_E_ARG
