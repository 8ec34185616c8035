"""One tensor split across ranks by root slices (one GPU per rank).

The nonzeros go to ranks by contiguous ranges of mode-`mode` slices holding
about nnz / world nonzeros each (a slice is never split), so the ranks'
trees are the trees of disjoint sub-tensors with the global dims. Factors
are replicated. A CP-ALS sweep runs mode by mode:

  * every rank computes its shard's MTTKRP of the mode (the memo plan works
    unchanged on the shard's own trees: an MTTKRP is linear in the nonzeros);
  * the ranks' MTTKRPs are summed (one all-reduce of dims[mode] x ldr FP64
    values);
  * every rank runs the same update from the sum (Gram inverse, A = M V^-1,
    normalisation, Gram, and for the last mode the fit's inner product), so
    the factors, Grams and lambda stay identical on every rank;
  * the fit follows from the replicated Grams and lambda with ||X||^2 summed
    once over the ranks.

The reference's only collective is the fit's MPI all-reduce
(adatm_cpd.c:147-157); the split here adds the MTTKRP sum. The collective is
the caller's: torch.distributed over NCCL for one GPU per rank
(`torch_allreduce`), or a local sum when one process holds several shards.
"""
from __future__ import annotations

import numpy as np


def partition_slices(inds, world, mode=0):
    """Rank of every nonzero: contiguous, nnz-balanced ranges of mode-`mode`
    slices (slice s goes to the rank whose share of the running nonzero count
    it completes or lies in)."""
    idx = np.asarray(inds[mode], dtype=np.int64)
    if world <= 1 or idx.size == 0:
        return np.zeros(idx.size, dtype=np.int64)
    counts = np.bincount(idx)
    cum = np.cumsum(counts)
    bounds = np.searchsorted(cum, [cum[-1] * k / world for k in range(1, world)], side="left")
    owner = np.searchsorted(bounds, np.arange(len(counts)), side="left")
    return owner[idx]


def shard_coo(inds, vals, world, rank, mode=0):
    """This rank's nonzeros (global indices and dims kept)."""
    keep = partition_slices(inds, world, mode) == rank
    return np.ascontiguousarray(np.asarray(inds)[:, keep]), np.ascontiguousarray(np.asarray(vals)[keep])


class ShardedCpd:
    """CP-ALS over shards.

    shards: objects with the shard interface of adatm_b200.Engine
      (mttkrp_into, update_from, fit_step, ttnorm, set_ttnorm, als_begin);
    buffers: buffers[s][m] is shard s's MTTKRP buffer of mode m, and
      pointer(buf) its device address;
    allreduce(bufs): replaces every buffer of the list by their sum;
    allreduce_scalar(x): the sum of x over the ranks.
    """

    def __init__(self, shards, nmodes, buffers, pointer, allreduce, allreduce_scalar=lambda x: x):
        self.shards = list(shards)
        self.nmodes = nmodes
        self.buffers = buffers
        self.pointer = pointer
        self.allreduce = allreduce
        self.allreduce_scalar = allreduce_scalar

    def begin(self):
        ttn = self.allreduce_scalar(sum(s.ttnorm() for s in self.shards))
        for s in self.shards:
            s.set_ttnorm(ttn)
            s.als_begin(graph=False)

    def sweep(self):
        for m in range(self.nmodes):
            for s, bufs in zip(self.shards, self.buffers):
                s.mttkrp_into(m, self.pointer(bufs[m]))
            self.allreduce([bufs[m] for bufs in self.buffers])
            for s, bufs in zip(self.shards, self.buffers):
                s.update_from(m, self.pointer(bufs[m]))
        fits = [s.fit_step() for s in self.shards]
        return fits[0]

    def als(self, niters, tol=0.0):
        """Sweeps until niters or |fit - previous| < tol (after the first);
        returns the fit trace."""
        self.begin()
        trace = []
        for it in range(niters):
            trace.append(self.sweep())
            if it > 0 and abs(trace[-1] - trace[-2]) < tol:
                break
        return trace


def torch_buffers(dims, rank_count, ldr, device):
    """One float64 device buffer per mode (dims[m] x ldr, the MTTKRP rows'
    FP64 sums) for each of rank_count local shards."""
    import torch
    return [[torch.zeros(int(d) * ldr, dtype=torch.float64, device=device) for d in dims]
            for _ in range(rank_count)]


def torch_allreduce(group=None):
    """The collective of one shard per rank: torch.distributed all_reduce
    (NCCL on GPUs), finished before the next update reads the buffer."""
    import torch
    import torch.distributed as dist

    def reduce(bufs):
        for b in bufs:
            dist.all_reduce(b, group=group)
        if bufs and bufs[0].is_cuda:
            torch.cuda.current_stream().synchronize()

    def reduce_scalar(x):
        t = torch.tensor([float(x)], dtype=torch.float64)
        if dist.get_backend(group) == "nccl":
            t = t.cuda()
        dist.all_reduce(t, group=group)
        return float(t.item())

    return reduce, reduce_scalar


def local_allreduce(bufs):
    """The collective of several shards in one process: every buffer
    becomes the sum of all (in shard order)."""
    total = bufs[0].clone()
    for b in bufs[1:]:
        total += b
    for b in bufs:
        b.copy_(total)
    if bufs[0].is_cuda:
        import torch
        torch.cuda.current_stream().synchronize()
