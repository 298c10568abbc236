"""GPU check of the domain decomposition (mhd_sub_* of the C ABI, driven by
magnetohydrodynamics_simulator_b200.decomposed): P x Q subdomains on one GPU exchanging their rings
through device buffers (LocalTransport) -- the ranks of a multi-GPU run emulated in one process --
against the single-domain context (mhd_step) and the C oracle on the same state.

Tolerances: dt to 1e-14 relative, fields to 1e-12 relative L-infinity (the decomposed solve adds
its dot products in another order), CG products within 1, |div B|_inf <= 1e-12.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle, default_alpha, rel_linf
from tests_helpers import smooth_state

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def m():
    import torch

    assert torch.cuda.is_available()
    import magnetohydrodynamics_simulator_b200 as mod

    assert mod.device_available(), "libmhd_b200.so has no kernels for this device"
    return mod


def _decomposed(m, nx, ny, dx, dy, eta, P, Q, ic, native=True):
    from magnetohydrodynamics_simulator_b200.decomposed import (DecomposedRun, GpuSubdomain,
                                                                LocalTransport, Partition)

    part = Partition(nx, ny, P, Q)
    subs = [GpuSubdomain(*part.shape(i), dx, dy, eta) for i in range(part.count)]
    run = DecomposedRun(part, LocalTransport(part, subs, native=native), dx, dy, eta)
    run.set_state(ic)
    return run, subs


@pytest.mark.parametrize("nx,ny,P,Q,steps,native", [(96, 80, 2, 2, 3, True), (70, 45, 3, 2, 2, True),
                                                    (128, 128, 2, 1, 3, True), (96, 80, 2, 2, 3, False)])
def test_decomposed_steps_match_single_context(m, nx, ny, P, Q, steps, native):
    """native: rings by mhd_sub_exchange_local; otherwise through mhd_sub_pack / mhd_sub_unpack
    buffers (the path strips take between GPUs)."""
    dx, dy = 2 * np.pi / nx, 1.6 * np.pi / ny
    eta = 0.02
    ic = smooth_state(nx, ny, dx, dy, seed=nx + ny)
    run, subs = _decomposed(m, nx, ny, dx, dy, eta, P, Q, ic, native=native)
    ctx = m.Context(nx, ny, dx, dy, eta)
    ctx.set_state(ic)
    orc = Oracle(nx, ny, dx, dy, eta)
    orc.set_state(ic)
    for _ in range(steps):
        dt_ctx = ctx.cfl_dt()
        dt, prods = run.step()
        assert abs(dt - dt_ctx) <= 1e-14 * dt_ctx, (dt, dt_ctx)
        ctx.step(dt)
        ctx.synchronize()
        want_prods = ctx.last_cg_products()
        assert all(abs(a - b) <= 1 for a, b in zip(prods, want_prods)), (prods, want_prods)
        orc.step(dt, alpha=default_alpha(dt, eta))
    assert run.status == "ok"
    got = run.get_state()
    for want in (ctx.get_state(), orc.get_state()):
        errs = [rel_linf(g, w, 1.0) for g, w in zip(got, want)]
        assert max(errs) <= 1e-12, errs
    rms, mx = run.divb()
    assert mx <= 1e-12
    assert abs(mx - ctx.divb()[1]) <= 1e-13
    ctx.close()
    for s in subs:
        s.close()


def test_decomposed_orszag_tang_matches_reference_goldens(m):
    """Orszag-Tang 128^2 split 2 x 2, the reference driver's dt sequence (first 20 steps of the
    golden run), against the single context stepped with the same dts."""
    from conftest import load_golden

    d = load_golden("ot128_ref.npz")
    n, dx, eta = int(d["nx"]), float(d["dx"]), float(d["eta"])
    ic = m.problems.orszag_tang(n, n, dx, dx)
    run, subs = _decomposed(m, n, n, dx, dx, eta, 2, 2, ic)
    ctx = m.Context(n, n, dx, dx, eta)
    ctx.set_state(ic)
    for dt in d["dts"][:20]:
        run.step(float(dt))
        ctx.step(float(dt))
    ctx.synchronize()
    errs = [rel_linf(g, w, 1.0) for g, w in zip(run.get_state(), ctx.get_state())]
    assert max(errs) <= 1e-12, errs
    assert run.divb()[1] <= 1e-12
    ctx.close()
    for s in subs:
        s.close()
