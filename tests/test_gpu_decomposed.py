"""GPU check of the domain decomposition (mhd_sub_* of the C ABI, driven by
magnetohydrodynamics_simulator_b200.decomposed): P x Q subdomains on one GPU exchanging their rings
through device buffers (LocalTransport) -- the ranks of a multi-GPU run emulated in one process --
against the single-domain context (mhd_step) and the C oracle on the same state.

The solve's decisions are taken on the device (mhd_subcg_*: each product one replayed CUDA graph
over the subdomains' streams) or on the host; in the same two-sweep form both must give the same
bits. With device decisions the default form is the single context's single-sweep solver on every
subdomain's interior.

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


_streams = []


def _decomposed(m, nx, ny, dx, dy, eta, P, Q, ic, native=True, shared=False, device=True, form=None):
    """shared: every subdomain on one stream; device: the solve's decisions on the device; form:
    the solve's form (None: the default)."""
    import torch
    from magnetohydrodynamics_simulator_b200.decomposed import (DecomposedRun, GpuSubdomain,
                                                                LocalTransport, Partition)

    part = Partition(nx, ny, P, Q)
    stream = None
    if shared:
        _streams.append(torch.cuda.Stream())
        stream = _streams[-1].cuda_stream
    subs = [GpuSubdomain(*part.shape(i), dx, dy, eta, stream=stream) for i in range(part.count)]
    run = DecomposedRun(part, LocalTransport(part, subs, native=native), dx, dy, eta,
                        device_decisions=device, cg_form=form)
    assert (run._group is not None) == device
    assert run.cg_form == (form or ("sweep" if device else "two_sweep"))
    run.set_state(ic)
    return run, subs


@pytest.mark.parametrize("nx,ny,P,Q,steps,native,shared,device,form", [
    (96, 80, 2, 2, 3, True, False, True, None), (70, 45, 3, 2, 2, True, False, True, None),
    (128, 128, 2, 1, 3, True, False, True, None), (96, 80, 2, 2, 3, False, False, True, None),
    (96, 80, 2, 2, 3, True, True, True, None), (96, 80, 1, 2, 3, True, False, True, None),
    (96, 80, 2, 2, 3, True, False, True, "two_sweep"), (70, 45, 3, 2, 2, True, False, False, None),
    (96, 80, 2, 2, 3, False, False, False, None)])
def test_decomposed_steps_match_single_context(m, nx, ny, P, Q, steps, native, shared, device, form):
    """native: rings by mhd_sub_exchange_local; otherwise through mhd_sub_pack / mhd_sub_unpack
    buffers (the path strips take between GPUs). shared: the subdomains on one stream. device:
    decisions on the device (with native rings: one graph per product). form: the solve's form."""
    dx, dy = 2 * np.pi / nx, 1.6 * np.pi / ny
    eta = 0.02
    ic = smooth_state(nx, ny, dx, dy, seed=nx + ny)
    run, subs = _decomposed(m, nx, ny, dx, dy, eta, P, Q, ic, native=native, shared=shared, device=device,
                            form=form)
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
    run.close()
    for s in subs:
        s.close()


def test_device_decisions_are_the_hosts(m):
    """Decisions on the device and on the host: the same dts, products and bits, over steps whose
    solves take several products."""
    nx, ny = 96, 80
    dx, dy = 2 * np.pi / nx, 1.6 * np.pi / ny
    eta = 0.05
    ic = smooth_state(nx, ny, dx, dy, seed=3)
    res = []
    for device in (True, False):
        run, subs = _decomposed(m, nx, ny, dx, dy, eta, 2, 2, ic, device=device, form="two_sweep")
        steps = [run.step() for _ in range(3)]
        res.append((steps, run.get_state(), run.status))
        run.close()
        for s in subs:
            s.close()
    assert res[0][0] == res[1][0]
    assert all(k > 1 for _, ks in res[0][0] for k in ks)
    assert res[0][2] == res[1][2] == "ok"
    for a, b in zip(res[0][1], res[1][1]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("nx,ny,P,Q", [(96, 80, 2, 2), (70, 45, 3, 2), (96, 80, 1, 2)])
def test_sweep_reading_neighbours_equals_sweep_reading_rings(m, nx, ny, P, Q):
    """The single-sweep solve's graphs read the cells around each interior from the neighbours'
    interiors; without graphs (rings through pack/unpack buffers) the same sweep reads its own
    rings. Both must give the same bits."""
    dx, dy = 2 * np.pi / nx, 1.6 * np.pi / ny
    eta = 0.04
    ic = smooth_state(nx, ny, dx, dy, seed=11)
    res = []
    for native in (True, False):
        run, subs = _decomposed(m, nx, ny, dx, dy, eta, P, Q, ic, native=native)
        steps = [run.step() for _ in range(3)]
        res.append((steps, run.get_state()))
        run.close()
        for s in subs:
            s.close()
    assert res[0][0] == res[1][0]
    for a, b in zip(res[0][1], res[1][1]):
        assert np.array_equal(a, b)


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


@pytest.mark.parametrize("form", ["sweep", "two_sweep"])
def test_decomposed_solve_edges_match_single_context(m, form):
    """A capped solve (2 products, not converged: the single-sweep form ends on an even iteration
    after k = 1 and on an odd one for the cap 3) and a zero right-hand side (eta = 0: x = 0, no
    product), against the single context with the same rules."""
    import torch
    from magnetohydrodynamics_simulator_b200.decomposed import (DecomposedRun, GpuSubdomain,
                                                                LocalTransport, Partition)

    nx, ny = 96, 80
    dx, dy = 2 * np.pi / nx, 1.6 * np.pi / ny
    ic = smooth_state(nx, ny, dx, dy, seed=9)
    for eta, cap in ((0.05, 2), (0.05, 3), (0.0, 0)):
        part = Partition(nx, ny, 2, 2)
        subs = [GpuSubdomain(*part.shape(i), dx, dy, eta) for i in range(part.count)]
        run = DecomposedRun(part, LocalTransport(part, subs), dx, dy, eta, cg_max_iters=cap, cg_form=form)
        run.set_state(ic)
        ctx = m.Context(nx, ny, dx, dy, eta, cg_max_iters=cap)
        ctx.set_state(ic)
        dt = ctx.cfl_dt()
        _, prods = run.step(dt)
        ctx.step(dt)
        assert ctx.synchronize_status() == (4 if cap else 0)  # MHD_ERR_CG_NOT_CONVERGED when capped
        want = ctx.last_cg_products()
        if cap:
            assert tuple(prods) == (cap, cap) == tuple(want), (prods, want)
            assert run.status == "cg_not_converged"
        else:
            assert tuple(prods) == (0, 0) == tuple(want)
            assert run.status == "ok"
        errs = [rel_linf(g, w, 1.0) for g, w in zip(run.get_state(), ctx.get_state())]
        assert max(errs) <= 1e-12, (eta, cap, errs)
        torch.cuda.synchronize()
        run.close()
        ctx.close()
        for s in subs:
            s.close()


NCCL_WORKER = r"""
import os, sys
sys.path.insert(0, {root!r})
sys.path.insert(0, os.path.join({root!r}, "tests"))
from datetime import timedelta
import numpy as np
import torch
import torch.distributed as dist
from magnetohydrodynamics_simulator_b200.decomposed import DecomposedRun, DistTransport, GpuSubdomain, Partition
from tests_helpers import smooth_state
torch.cuda.set_device(0)
dist.init_process_group("nccl", timeout=timedelta(seconds=60))
nx, ny, eta = {nx}, {ny}, {eta}
dx, dy = 2 * np.pi / nx, 1.6 * np.pi / ny
part = Partition(nx, ny, 1, 1)
out = {{}}
for dev in (True, False):
    sub = GpuSubdomain(nx, ny, dx, dy, eta)
    run = DecomposedRun(part, DistTransport(part, sub, device=torch.device("cuda")), dx, dy, eta,
                        device_decisions=dev)
    run.set_state(smooth_state(nx, ny, dx, dy, seed=4))
    steps = [run.step() for _ in range(3)]
    st = run.get_state()
    out[f"dts_{{dev}}"] = np.array([d for d, _ in steps])
    out[f"prods_{{dev}}"] = np.array([k for _, k in steps])
    out[f"form_{{dev}}"] = run.cg_form
    out[f"status_{{dev}}"] = run.status
    for k in range(6):
        out[f"f{{k}}_{{dev}}"] = st[k]
    run.close()
    sub.close()
torch.cuda.synchronize()
dist.barrier()
dist.destroy_process_group()
np.savez({out!r}, **out)
print("ok")
"""


def test_distributed_transport_one_nccl_rank_matches_single_context(m, tmp_path):
    """The DistTransport path on one GPU: one NCCL rank owning the whole grid (its rings come from
    itself), with the solve's decisions on the device (the sum slots all-gathered over NCCL on the
    subdomain's stream, the single-sweep form) and on the host (the two-sweep form), against the
    single context stepped with the same dts."""
    import os
    import socket
    import subprocess
    import sys

    from conftest import ROOT

    nx, ny, eta = 96, 80, 0.03
    out = str(tmp_path / "nccl1.npz")
    script = tmp_path / "worker.py"
    script.write_text(NCCL_WORKER.format(root=ROOT, nx=nx, ny=ny, eta=eta, out=out))
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0", MASTER_ADDR="127.0.0.1",
               MASTER_PORT=str(port), NCCL_NVLS_ENABLE="0")
    p = subprocess.run([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                       stderr=subprocess.STDOUT, text=True, timeout=300)
    assert p.returncode == 0, p.stdout[-3000:]
    d = np.load(out)
    dx, dy = 2 * np.pi / nx, 1.6 * np.pi / ny
    for dev in (True, False):
        assert str(d[f"form_{dev}"]) == ("sweep" if dev else "two_sweep")
        assert str(d[f"status_{dev}"]) == "ok"
        ctx = m.Context(nx, ny, dx, dy, eta)
        ctx.set_state(smooth_state(nx, ny, dx, dy, seed=4))
        for dt, k in zip(d[f"dts_{dev}"], d[f"prods_{dev}"]):
            assert abs(ctx.cfl_dt() - dt) <= 1e-14 * dt
            ctx.step(float(dt))
            ctx.synchronize()
            assert all(abs(a - b) <= 1 for a, b in zip(k, ctx.last_cg_products()))
        errs = [rel_linf(d[f"f{k}_{dev}"], w, 1.0) for k, w in enumerate(ctx.get_state())]
        assert max(errs) <= 1e-12, (dev, errs)
        ctx.close()


@pytest.mark.parametrize("device", [True, False])
def test_decomposed_solve_reports_nonfinite(m, device):
    """A NaN in one face of the field reaches the solve's right-hand side: the decomposed solve
    (decisions on the device or on the host) ends with status "nonfinite" after a fixed-dt step,
    as the single context reports MHD_ERR_NONFINITE for the same state."""
    nx, ny = 64, 48
    dx, dy = 2 * np.pi / nx, 2 * np.pi / ny
    eta = 0.05
    ic = smooth_state(nx, ny, dx, dy, seed=2)
    ic[4] = ic[4].copy()
    ic[4][30, 40] = np.nan  # bxf of a cell inside subdomain (1, 1) of the 2 x 2 split
    run, subs = _decomposed(m, nx, ny, dx, dy, eta, 2, 2, ic, device=device)
    run.step(1e-3)
    assert run.status == "nonfinite"
    # the CFL step of the same state (on the device with device decisions) flags it too
    run2, subs2 = _decomposed(m, nx, ny, dx, dy, eta, 2, 2, ic, device=device)
    run2.step()
    assert run2.status == "nonfinite"
    run2.close()
    for s in subs2:
        s.close()
    ctx = m.Context(nx, ny, dx, dy, eta)
    ctx.set_state(ic)
    ctx.step(1e-3)
    assert ctx.synchronize_status() == 3  # MHD_ERR_NONFINITE
    ctx.close()
    run.close()
    for s in subs:
        s.close()


def test_decomposed_orszag_tang_2048_matches_single_context(m):
    """At a benchmarked size: Orszag-Tang 2048^2 split 2 x 2 (the default single-sweep solve,
    decisions and CFL step on the device), 3 CFL steps against the single context on the same
    dts: 1e-12 relative per field, the same products, |div B|_inf <= 1e-12."""
    n = 2048
    dx = m.problems.grid_spacing(n)
    ic = m.problems.orszag_tang(n, n, dx, dx)
    run, subs = _decomposed(m, n, n, dx, dx, 1e-4, 2, 2, ic)
    ctx = m.Context(n, n, dx, dx, 1e-4)
    ctx.set_state(ic)
    for _ in range(3):
        dt, prods = run.step()
        assert abs(ctx.cfl_dt() - dt) <= 1e-14 * dt
        ctx.step(dt)
        ctx.synchronize()
        assert tuple(prods) == tuple(ctx.last_cg_products())
    assert run.status == "ok"
    errs = [rel_linf(g, w, 1.0) for g, w in zip(run.get_state(), ctx.get_state())]
    assert max(errs) <= 1e-12, errs
    assert run.divb()[1] <= 1e-12
    ctx.close()
    run.close()
    for s in subs:
        s.close()
