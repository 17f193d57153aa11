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


def test_means_without_allocation_beside_a_profiled_step(dcm):
    """A host thread that calls the allocation-free entry point while another
    thread runs a profiled dcm_step on a handle: the handle's launch counts
    and timed classes are exactly those of the same steps run alone (the
    other thread's launches are not counted into that handle's profile), and
    the means computed meanwhile are right."""
    import threading

    import torch

    c = small_bubble(ip=24, jp=20, kp=16)
    g = c.grid
    core = dcm.DynamicalCore(g)

    def profiled_steps():
        core.upload_state(c.state, c.dt, ptol=c.ptol, kord=c.kord, monotone=c.monotone)
        core.driver_start()
        core.profile(True)
        core.step(4)
        counts = {k: n for k, (_, n) in core.profile_read().items()}
        core.profile(False)
        return counts

    alone = profiled_steps()

    rng = np.random.default_rng(78)
    fields = [rand_field(g, rng) for _ in range(4)]
    expected = np.concatenate(core.horizontal_means(*fields)[:4])
    lib = dcm.library()
    dev = [torch.from_numpy(np.ravel(a, order="F").copy()).to("cuda") for a in fields]
    out = torch.empty(4 * (g.kp + 2), dtype=torch.float64, device="cuda")
    stream = torch.cuda.Stream()
    result = {}

    def run():
        result["counts"] = profiled_steps()

    t = threading.Thread(target=run)
    t.start()
    calls = 0
    while t.is_alive() or calls < 3:
        with torch.cuda.stream(stream):
            out.fill_(float("nan"))
        st = lib.dcm_horizontal_means_noalloc(
            g.ip, g.jp, g.kp, *[C.c_void_p(x.data_ptr()) for x in dev],
            C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert st == dcm.DCM_OK, st
        stream.synchronize()
        assert relerr(out.cpu().numpy(), expected) <= 1e-12
        calls += 1
    t.join()
    core.close()
    assert result["counts"] == alone, (result["counts"], alone)
