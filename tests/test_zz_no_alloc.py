"""The allocation-free resistive rate, mhd_resistive_rate_noalloc, against mhd_resistive_rate.

Some callers of this library cannot allocate device memory at the point where they need the
implicit resistive solve: plugins whose host application owns every device buffer, processes that
run under a fixed device-memory budget, and latency-sensitive loops that must not stall on the
device synchronisation cudaMalloc/cudaFree can imply. mhd_resistive_rate_noalloc serves them with
its scratch in one fixed-size device array; the caller passes only inputs and outputs.

These tests call it through the C ABI twice in a row (the array keeps the previous call's
contents) and compare both results with the context-based entry point's on the same input, within
the single-step tolerance of the parity tests (1e-12 relative L-infinity). They also check the
explicit path, that a call without a products pointer still reports the solve's status (an
iteration cap that is hit, a non-finite input), and that a grid beyond the array's capacity is
refused.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-12
NX, NY = 200, 160  # 32000 cells, within the 65536-cell capacity
ETA, ALPHA = 0.05, 2e-4


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def setup():
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
    dx, dy = 2 * np.pi / NX, 1.5 * np.pi / NY
    state = smooth_state(NX, NY, dx, dy, seed=5)
    bxf = torch.tensor(state[4], device="cuda")
    byf = torch.tensor(state[5], device="cuda")
    ctx = m.Context(NX, NY, dx, dy, ETA)
    p = capi.Params()
    assert lib.mhd_default_params(ctypes.byref(p), NX, NY, dx, dy, ETA) == 0
    yield dict(lib=lib, capi=capi, torch=torch, ctx=ctx, p=p, bxf=bxf, byf=byf, dx=dx, dy=dy)
    ctx.close()


def _context_rate(s, implicit):
    torch = s["torch"]
    want_x = torch.empty_like(s["bxf"])
    want_y = torch.empty_like(s["byf"])
    torch.cuda.synchronize()
    prods = s["ctx"].resistive_rate(s["bxf"].data_ptr(), s["byf"].data_ptr(), want_x.data_ptr(),
                                    want_y.data_ptr(), solve_implicitly=implicit, alpha=ALPHA)
    s["ctx"].synchronize()
    return prods, want_x.cpu().numpy(), want_y.cpu().numpy()


def _noalloc(s, implicit, params=None, bxf=None, with_products=True):
    torch = s["torch"]
    bxf = s["bxf"] if bxf is None else bxf
    out_x = torch.full_like(bxf, float("nan"))
    out_y = torch.full_like(s["byf"], float("nan"))
    torch.cuda.synchronize()
    prods = ctypes.c_longlong(-1)
    status = s["lib"].mhd_resistive_rate_noalloc(
        ctypes.byref(params or s["p"]), int(implicit), ALPHA, bxf.data_ptr(), s["byf"].data_ptr(),
        out_x.data_ptr(), out_y.data_ptr(), ctypes.byref(prods) if with_products else None, None)
    torch.cuda.synchronize()
    return status, prods.value, out_x.cpu().numpy(), out_y.cpu().numpy()


def test_noalloc_rate_matches_context_entry_point(setup):
    s = setup
    want_prods, wx, wy = _context_rate(s, implicit=True)
    assert want_prods > 0
    for _ in range(2):
        status, prods, gx, gy = _noalloc(s, implicit=True)
        assert status == 0, s["capi"].STATUS_NAMES.get(status, status)
        assert prods == want_prods  # same solver geometry as a context: same reduction order
        assert _rel(gx, wx) <= STEP_TOL
        assert _rel(gy, wy) <= STEP_TOL
    # without a products pointer: same result, status still returned
    status, _, gx, gy = _noalloc(s, implicit=True, with_products=False)
    assert status == 0
    assert _rel(gx, wx) <= STEP_TOL and _rel(gy, wy) <= STEP_TOL


def test_noalloc_explicit_rate_matches_context(setup):
    s = setup
    _, wx, wy = _context_rate(s, implicit=False)
    for _ in range(2):
        status, prods, gx, gy = _noalloc(s, implicit=False)
        assert status == 0 and prods == 0
        assert _rel(gx, wx) <= STEP_TOL and _rel(gy, wy) <= STEP_TOL


def test_noalloc_reports_failed_solves_without_products_pointer(setup):
    s = setup
    capi = s["capi"]
    capped = capi.Params()
    assert s["lib"].mhd_default_params(ctypes.byref(capped), NX, NY, s["dx"], s["dy"], ETA) == 0
    capped.cg_max_iters = 1
    status, _, _, _ = _noalloc(s, implicit=True, params=capped, with_products=False)
    assert status == 4  # MHD_ERR_CG_NOT_CONVERGED
    bad = s["bxf"].clone()
    bad[NY // 2, NX // 3] = float("nan")
    status, _, _, _ = _noalloc(s, implicit=True, bxf=bad, with_products=False)
    assert status == 3  # MHD_ERR_NONFINITE
    # the shared array is cleared per call: a good call afterwards succeeds and matches
    want_prods, wx, _ = _context_rate(s, implicit=True)
    status, prods, gx, _ = _noalloc(s, implicit=True)
    assert status == 0 and prods == want_prods and _rel(gx, wx) <= STEP_TOL


def test_noalloc_refuses_grids_beyond_capacity(setup):
    s = setup
    big = s["capi"].Params()
    assert s["lib"].mhd_default_params(ctypes.byref(big), 300, 300, s["dx"], s["dy"], ETA) == 0
    status = s["lib"].mhd_resistive_rate_noalloc(ctypes.byref(big), 1, ALPHA, s["bxf"].data_ptr(),
                                                 s["byf"].data_ptr(), s["bxf"].data_ptr(),
                                                 s["byf"].data_ptr(), None, None)
    assert status == 9  # MHD_ERR_TOO_LARGE
