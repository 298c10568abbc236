"""CPU checks of the domain-decomposition driver (magnetohydrodynamics_simulator_b200.decomposed):
the partition, the ring exchanges, the ordered reductions and the distributed conjugate gradient,
with a CPU stand-in for each subdomain (oracle/decomposed_oracle.py: the oracle's explicit rates
on the extended planes), against the single-domain C oracle step (oracle/mhd_oracle.c).

* in one process, 2 x 2 and 3 x 1 subdomains (LocalTransport);
* over two gloo ranks on 127.0.0.1, one subdomain per rank (DistTransport): a 2 x 1 and a 1 x 2
  split, so both axes exchange across ranks and along the other axis with themselves.

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


@pytest.mark.parametrize("P,Q", [(2, 2), (3, 1)])
def test_local_decomposition_matches_single_domain(P, Q):
    from magnetohydrodynamics_simulator_b200.decomposed import DecomposedRun, LocalTransport, Partition
    from oracle.decomposed_oracle import OracleSubdomain

    dx, dy = 2 * np.pi / NX, 1.7 * np.pi / NY
    ic = smooth_state(NX, NY, dx, dy, seed=21)
    part = Partition(NX, NY, P, Q)
    subs = [OracleSubdomain(*part.shape(i), dx, dy, ETA) for i in range(part.count)]
    run = DecomposedRun(part, LocalTransport(part, subs), dx, dy, ETA)
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
P, Q = {P}, {Q}
dist.init_process_group("gloo", timeout=timedelta(seconds=60))
rank = dist.get_rank()
dx, dy = 2 * np.pi / NX, 1.7 * np.pi / NY
ic = smooth_state(NX, NY, dx, dy, seed=21)
part = Partition(NX, NY, P, Q)
sub = OracleSubdomain(*part.shape(rank), dx, dy, ETA)
run = DecomposedRun(part, DistTransport(part, sub), dx, dy, ETA)
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


@pytest.mark.parametrize("P,Q", [(2, 1), (1, 2)])
def test_two_gloo_ranks_match_single_domain(tmp_path, P, Q):
    out = str(tmp_path / "rank0.npz")
    script = tmp_path / "worker.py"
    script.write_text(WORKER.format(root=ROOT, nx=NX, ny=NY, eta=ETA, P=P, Q=Q, out=out))
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
