"""CPU checks of the multi-rank plumbing of bench.py (replicas only: no collective on the data
path). Two gloo ranks on 127.0.0.1 agree on the slowest rank's time; a rank other than 0 of the
reference arm exits without work; the reference arm's replicas aggregate their throughput."""
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT

WORKER = r"""
import os, sys
sys.path.insert(0, {root!r})
import torch.distributed as dist
from datetime import timedelta
import bench
dist.init_process_group("gloo", timeout=timedelta(seconds=60))
rank = dist.get_rank()
t = bench.max_over_ranks(dist, 1.5 + rank, "cpu")
assert t == 1.5 + dist.get_world_size() - 1, t
assert bench.max_over_ranks(None, 3.0) == 3.0
dist.barrier()
dist.destroy_process_group()
print("ok", rank)
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_slowest_rank_time_over_gloo(tmp_path):
    script = tmp_path / "worker.py"
    script.write_text(WORKER.format(root=ROOT))
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT, text=True))
    outs = [p.communicate(timeout=120)[0] for p in procs]
    assert all(p.returncode == 0 for p in procs), outs
    assert "ok 0" in outs[0] and "ok 1" in outs[1]


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "3", "--warmup", "1"], env=env, capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "", (r.stdout, r.stderr)


def test_reference_replicas_aggregate():
    sys.path.insert(0, ROOT)
    import bench
    from oracle.oracle import reference_available

    if not reference_available():
        pytest.skip("oracle/_ref not built")
    rate, sec = bench.reference_replicas(32, 2, 0, 2)
    assert sec > 0 and rate == pytest.approx(2 * 32 * 32 * 2 / sec)
