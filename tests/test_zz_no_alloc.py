"""ugks_step_explicit_noalloc: the Explicit step for callers that cannot allocate device memory.

Host codes that own all device memory themselves (a pre-sized pool, a hard memory cap) or that
must not let cudaMalloc synchronise the device in their time loop cannot create a ugks_ctx.  This
entry point runs the same kernels on the caller's device arrays with its working arrays in a fixed
__device__ array.  It must agree with the context-based ugks_step_explicit, call after call.

Collected last (file name) so that a failure here comes after every other test has run.
"""
import ctypes

import numpy as np
import pytest

from ugks2d_high_order_b200.case import reference_case

pytestmark = pytest.mark.gpu

TOL = 1e-12   # the per-operator tolerance the other parity tests use (max|a-b| / max|b|)


def relmax(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300))


def test_noalloc_matches_context_path_two_calls_in_a_row(velocity):
    import torch
    from ugks2d_high_order_b200 import capi
    from ugks2d_high_order_b200.solver import Solver

    case = reference_case("Explicit")
    s = Solver(case, *velocity)
    s.init_freestream()
    h0, b0, W0 = s.download()

    dev = torch.device("cuda", 0)
    u, v, w = (torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in velocity)
    h = torch.from_numpy(h0.copy()).to(dev)
    b = torch.from_numpy(b0.copy()).to(dev)
    W = torch.from_numpy(W0.copy()).to(dev)
    torch.cuda.synchronize()
    L = capi.load()
    stream = torch.cuda.current_stream(dev).cuda_stream
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    dp = ctypes.POINTER(ctypes.c_double)

    for call in range(2):
        nsteps = 3 + call
        dt_c, res_c = s.step_explicit(nsteps)
        hc, bc, Wc = s.download()
        dt_n = np.zeros(1)
        res_n = np.zeros(4)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(dev)[0]
        rc = L.ugks_step_explicit_noalloc(ctypes.byref(s._params), vp(u), vp(v), vp(w), vp(h), vp(b), vp(W),
                                          nsteps, ctypes.c_void_p(stream), dt_n.ctypes.data_as(dp),
                                          res_n.ctypes.data_as(dp))
        assert rc == capi.UGKS_OK, f"call {call}: {L.ugks_error_string(rc).decode()}"
        torch.cuda.synchronize()
        if call > 0:   # the first call may load the library's scratch array; later calls take nothing
            assert torch.cuda.mem_get_info(dev)[0] == free_before, "a repeated call changed the free device memory"
        assert relmax(h.cpu().numpy(), hc) <= TOL, call
        assert relmax(b.cpu().numpy(), bc) <= TOL, call
        assert relmax(W.cpu().numpy(), Wc) <= TOL, call
        assert abs(dt_n[0] - dt_c) <= TOL * dt_c
        assert np.allclose(res_n, res_c, rtol=1e-9, atol=0)
    s.close()


def test_noalloc_rejects_oversized_problem(velocity):
    import torch
    from ugks2d_high_order_b200 import capi
    from ugks2d_high_order_b200.solver import Solver

    case = reference_case("Explicit")
    s = Solver(case, *velocity)
    p = capi.UgksParams.from_buffer_copy(s._params)
    p.ny = 4096   # 8 x 4096 cells x 1024 velocities needs far more than the fixed array
    p.dy = 1.0 / 4096
    dev = torch.device("cuda", 0)
    t = torch.zeros(4, dtype=torch.float64, device=dev)
    L = capi.load()
    vp = ctypes.c_void_p(t.data_ptr())
    rc = L.ugks_step_explicit_noalloc(ctypes.byref(p), vp, vp, vp, vp, vp, vp, 1, None, None, None)
    assert rc == capi.UGKS_EINVAL
    s.close()
