"""Batched CP-ALS sweeps of many uneven tensors (the 64-tensor workload).

    python -m adatm_b200.batch_case [--tensors 64] [--sweeps 20] [--no-tune] [--model MODEL.npz]
                                    [--fp64-check]

Tensor k (seed k): order uniform in {3, 4, 5}, every dim log-uniform in
[100, 50000], nnz drawn log-uniform in [10,000, 2,000,000], indices uniform
or Zipf(alpha in [1.0, 1.5]) chosen by the seed, values U(0, 1), R = 16,
FP32. Each tensor gets its plan (the learned plan model when given, else the
analytic model) and, unless --no-tune, its chunk sizes from the autotuner.
Reported: ms per ALS iteration of all tensors, (a) one CUDA graph per tensor
launched one after another, (b) the batched graph (every tensor on its own
branch), plus the fits of both runs and of a second batched run from the same
start (deterministic accumulation: they agree bit for bit). --fp64-check also
runs every tensor's ALS in FP64 on the host (the reference's ALS steps with
the oracle's COO MTTKRP, test infrastructure) and reports each fit's distance
from it.
"""
import argparse
import json
import math

import numpy as np

import adatm_b200 as A

RANK = 16


def spec(k):
    rng = np.random.default_rng(k)
    N = int(rng.integers(3, 6))
    dims = [int(round(math.exp(rng.uniform(math.log(100), math.log(50000))))) for _ in range(N)]
    nnz = int(round(math.exp(rng.uniform(math.log(1e4), math.log(2e6)))))
    alpha = float(rng.uniform(1.0, 1.5)) if rng.uniform() < 0.5 else None
    return N, dims, nnz, alpha


def build(n, tune, model):
    tensors, engines, tuned = [], [], []
    for k in range(n):
        N, dims, nnz, alpha = spec(k)
        t = A.Tensor.generate(dims, nnz, alpha=alpha, seed=k)
        plan = A.plan_learned(t, RANK, model)[0] if model else A.plan_analytic(t, RANK)[0]
        e = A.Engine(t, RANK, plan)
        tuned.append(e.autotune() if tune else -1)
        tensors.append(t)
        engines.append(e)
    return tensors, engines, tuned


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--tensors", type=int, default=64)
    ap.add_argument("--sweeps", type=int, default=20)
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--model", default=None)
    ap.add_argument("--fp64-check", action="store_true")
    a = ap.parse_args()
    A.lib().adatm_set_device(0)
    model = A.PlanModel.load(a.model) if a.model else None
    tensors, engines, tuned = build(a.tensors, not a.no_tune, model)
    # (a) one graph per tensor, one after another
    for e in engines:
        e.init_factors(0)
        e.als_begin(graph=True)
    for e in engines:
        e.time_sweeps(2)
    seq = sum(e.time_sweeps(a.sweeps) for e in engines) / a.sweeps
    seq_fit = [e.fit() for e in engines]
    # the same sequential run again (deterministic accumulation: the same fits)
    for e in engines:
        e.init_factors(0)
        e.als_begin(graph=True)
        e.time_sweeps(2 + a.sweeps)
    rerun_fit = [e.fit() for e in engines]
    # (b) the batched graph, from the same start
    for e in engines:
        e.init_factors(0)
    b = A.BatchSweep(engines)
    b.begin()
    b.time_sweeps(2)
    bat = b.time_sweeps(a.sweeps) / a.sweeps
    bat_fit = [e.fit() for e in engines]
    # the batch again from the same start: the same fits, bit for bit
    for e in engines:
        e.init_factors(0)
    b.begin()
    b.time_sweeps(2 + a.sweeps)
    bat_fit2 = [e.fit() for e in engines]
    out = {"tensors": a.tensors, "rank": RANK, "nnz_total": int(sum(t.info()[1] for t in tensors)),
           "orders": [t.info()[0] for t in tensors], "sweeps": a.sweeps,
           "ms_per_iteration_sequential_graphs": seq, "ms_per_iteration_batched_graph": bat,
           "speedup": seq / bat, "kernels_per_iteration": b.kernels(),
           "autotuned_option": tuned, "plan_model": a.model or "analytic",
           "max_fit_difference": float(np.max(np.abs(np.array(seq_fit) - np.array(bat_fit)))),
           "max_fit_difference_sequential_rerun":
               float(np.max(np.abs(np.array(seq_fit) - np.array(rerun_fit)))),
           "batched_reruns_identical": bat_fit == bat_fit2}
    if a.fp64_check:
        import oracle as O
        dev = []
        for t, f in zip(tensors, bat_fit):
            inds, vals, dims = t.download()
            start = [np.asarray(m, dtype=np.float32).astype(np.float64)
                     for m in O.init_factors(dims, RANK, 0)]
            ref = O.cpd_als_coo(inds, vals, dims, RANK, start, 2 + a.sweeps, 0.0)["fit"]
            dev.append(abs(f - ref))
        out["fp64_fit_distance"] = {"max": float(np.max(dev)), "mean": float(np.mean(dev)),
                                    "over_1e-4": int(np.sum(np.array(dev) > 1e-4))}
    print(json.dumps(out))
    b.free()


if __name__ == "__main__":
    main()
