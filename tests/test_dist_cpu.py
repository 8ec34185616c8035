"""The multi-rank plumbing of bench.py (one replica per rank: barrier,
max-over-ranks timing, whole-job aggregate) on two gloo ranks on the CPU."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import os, sys
sys.path.insert(0, {root!r})
import bench
world, rank, local = bench.dist_setup(backend="gloo")
assert world == 2 and rank in (0, 1)
bench.barrier(world)
m = bench.max_over_ranks(10.0 + 5.0 * rank, world)
assert m == 15.0, m
v = bench.replica_ms_per_sweep(m, 3, world)
assert abs(v - 15.0 / 6.0) < 1e-12
bench.barrier(world)
import torch.distributed as dist
dist.destroy_process_group()
print("rank", rank, "ok")
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_barrier_and_max():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, WORLD_SIZE="2", RANK=str(rank), LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER.format(root=ROOT)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
    outs = []
    for p in procs:
        try:
            out, _ = p.communicate(timeout=120)
        except subprocess.TimeoutExpired:
            p.kill()
            pytest.fail("gloo rank did not finish")
        outs.append(out)
        assert p.returncode == 0, out
    assert all("ok" in o for o in outs)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.replica_ms_per_sweep(12.0, 4, 1) == 3.0
