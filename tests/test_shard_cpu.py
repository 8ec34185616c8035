"""One tensor split across two gloo ranks on the CPU (adatm_b200.shard):
nnz-balanced root-slice partitions, the per-mode MTTKRP sum, replicated
updates; each rank's shard computed by the FP64 oracle. The 2-rank fit
trace equals the 1-rank FP64 run."""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from adatm_b200 import shard as S  # noqa: E402

WORKER = r"""
import os, sys
sys.path.insert(0, {root!r}); sys.path.insert(0, {tests!r})
import numpy as np, torch, torch.distributed as dist
import oracle as O
from adatm_b200 import shard as S
from _oracle_shard import OracleShard
dist.init_process_group("gloo")
world, rank = dist.get_world_size(), dist.get_rank()
inds, vals, dims = O.generate([400, 300, 200, 100], 150000, alpha=1.2, seed=3)
R = 8
li, lv = S.shard_coo(inds, vals, world, rank)
sh = OracleShard(li, lv, dims, R)
bufs = [[torch.zeros(d * R, dtype=torch.float64) for d in dims]]
reduce, reduce_scalar = S.torch_allreduce()
cpd = S.ShardedCpd([sh], len(dims), bufs, lambda b: b, reduce, reduce_scalar)
trace = cpd.als(6)
ref = O.cpd_als_coo(inds, vals, dims, R, O.init_factors(dims, R, 0), 6, 0.0)["trace"]
assert np.max(np.abs(np.array(trace) - ref)) < 1e-9, (trace, ref)
n = torch.tensor([float(len(lv))], dtype=torch.float64)
dist.all_reduce(n)
assert int(n.item()) == len(vals)
dist.destroy_process_group()
print("rank", rank, "ok", len(lv), trace[-1])
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_sharded_cpd_equals_one_rank():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, WORLD_SIZE="2", RANK=str(rank), LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), OMP_NUM_THREADS="2")
        code = WORKER.format(root=ROOT, tests=os.path.join(ROOT, "tests"))
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT, text=True))
    outs = []
    for p in procs:
        try:
            out, _ = p.communicate(timeout=300)
        except subprocess.TimeoutExpired:
            p.kill()
            pytest.fail("gloo rank did not finish")
        outs.append(out)
        assert p.returncode == 0, out
    assert all("ok" in o for o in outs)
    sizes = [int(o.split("ok")[1].split()[0]) for o in outs]
    assert min(sizes) > 0.3 * sum(sizes)   # nnz-balanced (Zipf slices)


@pytest.mark.parametrize("world", [1, 2, 3, 5])
def test_partition_covers_and_balances(world):
    rng = np.random.default_rng(world)
    idx = rng.integers(0, 1000, 50000)
    inds = np.stack([idx, rng.integers(0, 50, 50000)])
    own = S.partition_slices(inds, world)
    assert own.min() >= 0 and own.max() <= world - 1
    # a slice is never split, ranges are contiguous in slice order
    for s in np.unique(idx)[:200]:
        assert len(np.unique(own[idx == s])) == 1
    order = np.argsort(idx, kind="stable")
    assert np.all(np.diff(own[order]) >= 0)
    counts = np.bincount(own, minlength=world)
    assert counts.max() - counts.min() <= 2 * np.bincount(idx).max() + 1


def test_local_shards_sum_like_one_rank():
    """Several shards in one process (local sum) give the 1-rank trace."""
    import torch
    import oracle as O
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from _oracle_shard import OracleShard
    inds, vals, dims = O.generate([300, 200, 100, 60], 60000, alpha=1.1, seed=4)
    R = 6
    shards, bufs = [], []
    for r in range(3):
        li, lv = S.shard_coo(inds, vals, 3, r)
        shards.append(OracleShard(li, lv, dims, R))
        bufs.append([torch.zeros(d * R, dtype=torch.float64) for d in dims])
    cpd = S.ShardedCpd(shards, len(dims), bufs, lambda b: b, S.local_allreduce)
    trace = cpd.als(5)
    ref = O.cpd_als_coo(inds, vals, dims, R, O.init_factors(dims, R, 0), 5, 0.0)["trace"]
    assert np.max(np.abs(np.array(trace) - ref)) < 1e-9
