"""CPU checks of the domain-decomposition driver (magnetohydrodynamics_simulator_b200.decomposed):
the partition, the ring exchanges, the ordered reductions and the distributed conjugate gradient,
with a CPU stand-in for each subdomain (oracle/decomposed_oracle.py: the oracle's explicit rates
on the extended planes), against the single-domain C oracle step (oracle/mhd_oracle.c).

* in one process, 2 x 2 and 3 x 1 subdomains (LocalTransport);
* over two gloo ranks on 127.0.0.1, one subdomain per rank (DistTransport): a 2 x 1 and a 1 x 2
  split, so both axes exchange across ranks and along the other axis with themselves;
* the solve's decisions in a control block (the library's rules, mhd_subcg_decide_host) against
  the host's decisions: bit-identical states and products, and the rules' edge cases.

Tolerances: dt to 1e-14 relative, fields to 1e-12 relative L-infinity (the stand-in sums the
decomposed dot products in another order than the oracle's CG, and forms the stages in the GPU's
split), CG products within 1.
"""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT
from oracle.oracle import Oracle, default_alpha, rel_linf
from tests_helpers import smooth_state

NX, NY = 36, 28
ETA = 0.05


def _reference_run(ic, dx, dy, steps):
    orc = Oracle(NX, NY, dx, dy, ETA)
    orc.set_state(ic)
    dts, prods = [], []
    for _ in range(steps):
        dt = orc.cfl_dt()
        prods.append(orc.step(dt, alpha=default_alpha(dt, ETA)))
        dts.append(dt)
    return orc.get_state(), np.array(dts), np.array(prods), orc.divb()


def _check(got, dts, prods, want, want_dts, want_prods):
    assert np.max(np.abs(np.array(dts) - want_dts) / want_dts) <= 1e-14
    assert np.max(np.abs(np.array(prods) - want_prods)) <= 1, (prods, want_prods)
    errs = [rel_linf(g, w, 1.0) for g, w in zip(got, want)]
    assert max(errs) <= 1e-12, errs


@pytest.mark.parametrize("P,Q,device_decisions", [(2, 2, True), (3, 1, True), (2, 2, False)])
def test_local_decomposition_matches_single_domain(P, Q, device_decisions):
    from magnetohydrodynamics_simulator_b200.decomposed import DecomposedRun, LocalTransport, Partition
    from oracle.decomposed_oracle import OracleSubdomain

    dx, dy = 2 * np.pi / NX, 1.7 * np.pi / NY
    ic = smooth_state(NX, NY, dx, dy, seed=21)
    part = Partition(NX, NY, P, Q)
    subs = [OracleSubdomain(*part.shape(i), dx, dy, ETA) for i in range(part.count)]
    run = DecomposedRun(part, LocalTransport(part, subs), dx, dy, ETA, device_decisions=device_decisions)
    assert (run._group is not None) == device_decisions
    run.set_state(ic)
    dts, prods = [], []
    for _ in range(3):
        dt, k = run.step()
        dts.append(dt)
        prods.append(k)
    want, want_dts, want_prods, want_divb = _reference_run(ic, dx, dy, 3)
    _check(run.get_state(), dts, prods, want, want_dts, want_prods)
    assert run.status == "ok"
    rms, mx = run.divb()
    assert abs(mx - want_divb[1]) <= 1e-12 and abs(rms - want_divb[0]) <= 1e-12


def test_control_block_decisions_are_the_hosts():
    """The same 3 CFL steps with the decisions in a control block and on the host: identical bits."""
    from magnetohydrodynamics_simulator_b200.decomposed import DecomposedRun, LocalTransport, Partition
    from oracle.decomposed_oracle import OracleSubdomain

    dx, dy = 2 * np.pi / NX, 1.7 * np.pi / NY
    ic = smooth_state(NX, NY, dx, dy, seed=5)
    part = Partition(NX, NY, 2, 2)
    res = []
    for mode, lag in ((True, 1), (False, 1), (True, 3)):
        subs = [OracleSubdomain(*part.shape(i), dx, dy, ETA) for i in range(part.count)]
        run = DecomposedRun(part, LocalTransport(part, subs), dx, dy, ETA, device_decisions=mode,
                            poll_lag=lag)
        run.set_state(ic)
        steps = [run.step() for _ in range(3)]
        res.append((steps, run.get_state()))
    for other in res[1:]:
        assert res[0][0] == other[0]
        for a, b in zip(res[0][1], other[1]):
            assert np.array_equal(a, b)


def test_control_block_rules():
    """mhd_subcg_decide_host: Eigen's rules over the slots added in order (zero and non-finite
    right-hand sides, the threshold, the product cap, alpha and beta)."""
    import ctypes

    from magnetohydrodynamics_simulator_b200.capi import load_library
    from magnetohydrodynamics_simulator_b200.decomposed import HostCgGroup, _bind

    lib = _bind(load_library())
    g = HostCgGroup(lib, 3)

    def run(phase, sums, tol=1e-3, maxp=3):
        for i, v in enumerate(sums):
            g.slot(i)[:len(v)] = v
        g.decide(phase, tol, maxp)
        return g.ctl.copy()

    c = run(0, [[0.0, 0.0]] * 3)
    assert c[0] == 0.0 and c[1] == 0 and c[2] == 0  # b = 0: no product
    c = run(0, [[1.0, 0.5], [np.nan, 0.0], [1.0, 0.5]])
    assert c[0] == 0.0 and c[1] == 2  # non-finite right-hand side
    c = run(0, [[1.0, 0.5], [2.0, 0.25], [4.0, 1.0]])
    assert c[0] == 1.0 and c[3] == 7.0 and c[5] == 1.75 and c[4] == 1e-3 * 1e-3 * 7.0
    c = run(1, [[0.5], [0.25], [0.125]])
    assert c[6] == 1.75 / 0.875  # alpha = r.z / p.q
    c = run(2, [[1.0, 0.7], [1.0, 0.0], [1.0, 0.0]])
    assert c[0] == 1.0 and c[2] == 1 and c[7] == 0.7 / 1.75 and c[5] == 0.7  # beta, new r.z
    c = run(2, [[1e-7, 0.1], [0.0, 0.0], [0.0, 0.0]])
    assert c[0] == 0.0 and c[1] == 0 and c[2] == 2  # converged: |r|^2 below tol^2 |b|^2
    run(0, [[1.0, 1.0], [1.0, 1.0], [1.0, 1.0]])
    for k in range(3):
        run(1, [[1.0], [0.0], [0.0]])
        c = run(2, [[1.0, 1.0], [0.0, 0.0], [0.0, 0.0]])
    assert c[0] == 0.0 and c[1] == 1 and c[2] == 3  # the product cap: not converged
    c = run(2, [[1.0, 1.0]] * 3)
    assert c[2] == 3  # an ended solve takes no further decision
    assert lib.mhd_subcg_decide_host(None, g.slots.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                     3, 0, 1e-3, 3) != 0

    # the single-sweep form: phase 3 after the right-hand side (|b|^2, b.z, z.Az), 4 after an
    # iteration (r.r, r.z, z.Az, z.q) with p.Ap by its recurrence
    c = run(3, [[1.0, 0.5, 0.25], [2.0, 0.25, 0.25], [4.0, 1.0, 0.5]])
    assert c[0] == 1.0 and c[3] == 7.0 and c[5] == 1.75 and c[9] == 1.0 and c[6] == 1.75
    assert c[11] == -1.0 and c[13] == 0.0
    c = run(4, [[1.0, 0.7, 0.5, 0.25], [0.0, 0.0, 0.0, 0.0], [0.0, 0.0, 0.0, 0.0]])
    beta = 0.7 / 1.75
    pap = 0.5 + 2.0 * beta * 0.25 + beta * beta * 1.0
    assert c[0] == 1.0 and c[2] == 1 and c[11] == 0 and c[12] == 1.75 and c[7] == beta
    assert c[9] == pap and c[10] == 1.75 and c[6] == 0.7 / pap
    c = run(4, [[1.0, 0.7, -10.0, 0.0], [0.0] * 4, [0.0] * 4])
    assert c[0] == 0.0 and c[1] == 2 and c[13] == 1.0  # p.Ap <= 0: breakdown, x = 0
    c = run(3, [[0.0, 0.0, 0.0]] * 3)
    assert c[0] == 0.0 and c[13] == 1.0 and c[1] == 0  # zero right-hand side


def test_partition_sizes_and_neighbours():
    from magnetohydrodynamics_simulator_b200.decomposed import EAST, NORTH, SOUTH, WEST, Partition

    part = Partition(37, 29, 3, 2)
    assert part.xs == [13, 12, 12] and part.ys == [15, 14]
    assert part.x0 == [0, 13, 25] and part.y0 == [0, 15]
    assert part.neighbour(0, WEST) == 2 and part.neighbour(2, EAST) == 0
    assert part.neighbour(0, SOUTH) == 3 and part.neighbour(4, NORTH) == 1
    with pytest.raises(ValueError):
        Partition(12, 12, 4, 1)  # 3-cell subdomains cannot hold a 4-cell ring


WORKER = r"""
import os, sys
sys.path.insert(0, {root!r})
sys.path.insert(0, os.path.join({root!r}, "tests"))
import numpy as np
import torch.distributed as dist
from datetime import timedelta
from magnetohydrodynamics_simulator_b200.decomposed import DecomposedRun, DistTransport, Partition
from oracle.decomposed_oracle import OracleSubdomain
from tests_helpers import smooth_state
NX, NY, ETA = {nx}, {ny}, {eta}
P, Q, DEV = {P}, {Q}, {dev}
dist.init_process_group("gloo", timeout=timedelta(seconds=60))
rank = dist.get_rank()
dx, dy = 2 * np.pi / NX, 1.7 * np.pi / NY
ic = smooth_state(NX, NY, dx, dy, seed=21)
part = Partition(NX, NY, P, Q)
sub = OracleSubdomain(*part.shape(rank), dx, dy, ETA)
run = DecomposedRun(part, DistTransport(part, sub), dx, dy, ETA, device_decisions=DEV)
run.set_state(ic)
dts, prods = [], []
for _ in range(3):
    dt, k = run.step()
    dts.append(dt); prods.append(k)
state = run.get_state()
divb = run.divb()
if rank == 0:
    np.savez({out!r}, dts=np.array(dts), prods=np.array(prods), divb=np.array(divb), status=run.status,
             **{{f"f{{k}}": state[k] for k in range(6)}})
dist.barrier()
dist.destroy_process_group()
print("ok", rank)
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("P,Q,dev", [(2, 1, True), (1, 2, False)])
def test_two_gloo_ranks_match_single_domain(tmp_path, P, Q, dev):
    out = str(tmp_path / "rank0.npz")
    script = tmp_path / "worker.py"
    script.write_text(WORKER.format(root=ROOT, nx=NX, ny=NY, eta=ETA, P=P, Q=Q, dev=dev, out=out))
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT, text=True))
    outs = [p.communicate(timeout=300)[0] for p in procs]
    assert all(p.returncode == 0 for p in procs), outs
    d = np.load(out)
    dx, dy = 2 * np.pi / NX, 1.7 * np.pi / NY
    ic = smooth_state(NX, NY, dx, dy, seed=21)
    want, want_dts, want_prods, want_divb = _reference_run(ic, dx, dy, 3)
    _check([d[f"f{k}"] for k in range(6)], d["dts"], d["prods"], want, want_dts, want_prods)
    assert str(d["status"]) == "ok"
    assert abs(d["divb"][1] - want_divb[1]) <= 1e-12


def test_gpu_subdomain_refuses_without_device():
    """The product's subdomain needs the CUDA library and a device: no CPU fallback."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from magnetohydrodynamics_simulator_b200.capi import MHDError
    from magnetohydrodynamics_simulator_b200.decomposed import GpuSubdomain

    with pytest.raises(MHDError):
        GpuSubdomain(16, 16, 0.1, 0.1, 0.01)
    from magnetohydrodynamics_simulator_b200.capi import load_library
    from magnetohydrodynamics_simulator_b200.decomposed import DeviceCgGroup, _bind

    lib = _bind(load_library())
    with pytest.raises(MHDError):
        DeviceCgGroup(lib, 4, 0)  # the device decision group too
    # argument checks of the device entry points come before any device call
    assert lib.mhd_sub_cg_sweep_iter_dev(None, None, None) != 0
    assert lib.mhd_subcg_sweep_product(None, None, 2, 2, 1e-3, 10, 0, 1) != 0
    assert lib.mhd_subcg_decide_on(None, None, 0, 1e-3, 10) != 0
