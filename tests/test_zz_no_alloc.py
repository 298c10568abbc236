"""The allocation-free resistive rate, mhd_resistive_rate_noalloc, against mhd_resistive_rate.

Some callers of this library cannot allocate device memory at the point where they need the
implicit resistive solve: plugins whose host application owns every device buffer, processes that
run under a fixed device-memory budget, and latency-sensitive loops that must not stall on the
device synchronisation cudaMalloc/cudaFree can imply. mhd_resistive_rate_noalloc serves them with
its scratch in one fixed-size device array; the caller passes only inputs and outputs.

This test calls it through the C ABI twice in a row (the array keeps the previous call's contents)
and compares both results with the context-based entry point's on the same input, within the
single-step tolerance of the parity tests (1e-12 relative L-infinity), and checks that a grid
beyond the array's capacity is refused.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-12


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_noalloc_rate_matches_context_entry_point():
    import torch

    import magnetohydrodynamics_simulator_b200 as m
    from magnetohydrodynamics_simulator_b200 import capi
    from tests_helpers import smooth_state

    assert torch.cuda.is_available()
    lib = capi.load_library()
    vp = ctypes.c_void_p
    lib.mhd_resistive_rate_noalloc.argtypes = [ctypes.POINTER(capi.Params), ctypes.c_int,
                                               ctypes.c_double, vp, vp, vp, vp,
                                               ctypes.POINTER(ctypes.c_longlong), vp]
    nx, ny = 200, 160  # 32000 cells, within the 65536-cell capacity
    dx, dy = 2 * np.pi / nx, 1.5 * np.pi / ny
    eta, alpha = 0.05, 2e-4
    state = smooth_state(nx, ny, dx, dy, seed=5)
    bxf = torch.tensor(state[4], device="cuda")
    byf = torch.tensor(state[5], device="cuda")

    # the existing entry point (context workspace)
    ctx = m.Context(nx, ny, dx, dy, eta)
    want_x = torch.empty_like(bxf)
    want_y = torch.empty_like(byf)
    torch.cuda.synchronize()
    want_prods = ctx.resistive_rate(bxf.data_ptr(), byf.data_ptr(), want_x.data_ptr(),
                                    want_y.data_ptr(), solve_implicitly=True, alpha=alpha)
    ctx.synchronize()
    assert want_prods > 0
    wx, wy = want_x.cpu().numpy(), want_y.cpu().numpy()

    p = capi.Params()
    assert lib.mhd_default_params(ctypes.byref(p), nx, ny, dx, dy, eta) == 0
    for _ in range(2):
        out_x = torch.full_like(bxf, float("nan"))
        out_y = torch.full_like(byf, float("nan"))
        torch.cuda.synchronize()
        prods = ctypes.c_longlong(-1)
        status = lib.mhd_resistive_rate_noalloc(ctypes.byref(p), 1, alpha, bxf.data_ptr(),
                                                byf.data_ptr(), out_x.data_ptr(), out_y.data_ptr(),
                                                ctypes.byref(prods), None)
        assert status == 0, capi.STATUS_NAMES.get(status, status)
        torch.cuda.synchronize()
        assert prods.value == want_prods
        assert _rel(out_x.cpu().numpy(), wx) <= STEP_TOL
        assert _rel(out_y.cpu().numpy(), wy) <= STEP_TOL

    # a grid beyond the fixed scratch is refused with its own status
    big = capi.Params()
    assert lib.mhd_default_params(ctypes.byref(big), 300, 300, dx, dy, eta) == 0
    status = lib.mhd_resistive_rate_noalloc(ctypes.byref(big), 1, alpha, bxf.data_ptr(),
                                            byf.data_ptr(), out_x.data_ptr(), out_y.data_ptr(),
                                            None, None)
    assert status == 9  # MHD_ERR_TOO_LARGE
