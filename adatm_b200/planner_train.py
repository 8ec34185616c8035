"""Learned plan model: timed training data, GPU training, regret evaluation.

    python -m adatm_b200.planner_train make  --tensors 400 --seed0 1000 --out DATA.npz
    python -m adatm_b200.planner_train train --data DATA.npz --model MODEL.npz
    python -m adatm_b200.planner_train eval  --model MODEL.npz [--big]

`make` draws seeded synthetic tensors (order --min-order..8, dims
log-uniform in [50, 100000], nnz log-uniform in [--min-nnz, --max-nnz], Zipf
alpha uniform in [1.0, 1.6], values U(0, 1), R drawn from --ranks),
enumerates the candidate plans of
decide_candidate_configs, and times a CP-ALS sweep of every candidate with the
library's own kernels (CUDA-graph replays, CUDA events): the label of a
(tensor, candidate) row is log10(ms per sweep). The analytic model's choice is
kept beside it.

`train` (one or more --data sets) standardises the features, holds out the
last 20% of every set's tensors, trains
the network on the GPU (the library's forward, backward and Adam kernels) to
regress the label, and reports the regret of the learned and the analytic
choice on the held-out tensors: regret = time(chosen) / time(best) - 1, the
best found by exhaustive timing.

`eval --big` times every candidate on the 6th-order held-out tensor
50000x20000x10000x2000x500x100, 100M Zipf(1.3) draws, R = 32, and reports the
three choices.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys

import numpy as np

import adatm_b200 as A

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_MODEL = os.path.join(HERE, "planner_data", "plan_model.npz")
WIDTHS = [A.PLAN_FEATURES, 64, 64, 1]
RANK = 32


def draw_tensor_spec(seed, max_nnz, min_nnz=1e5, min_order=4, ranks=(RANK,)):
    rng = np.random.default_rng(seed)
    N = int(rng.integers(min_order, 9))
    dims = [int(round(math.exp(rng.uniform(math.log(50), math.log(100000))))) for _ in range(N)]
    nnz = int(round(math.exp(rng.uniform(math.log(min_nnz), math.log(max_nnz)))))
    alpha = float(rng.uniform(1.0, 1.6))
    R = int(ranks[int(rng.integers(0, len(ranks)))]) if len(ranks) > 1 else int(ranks[0])
    return N, dims, nnz, alpha, R


def time_plan(t, plan, sweeps=5, R=RANK):
    e = A.Engine(t, R, plan)
    try:
        e.init_factors(0)
        e.als_begin(graph=True)
        e.time_sweeps(2)
        return e.time_sweeps(sweeps) / sweeps
    finally:
        e.free()


def measure_tensor(t, sweeps=5, R=RANK):
    """Features, exact bytes, candidates, per-candidate ms and the analytic
    choice for one tensor."""
    X, nbytes, cands = A.plan_features(t, R)
    _, _, chosen = A.plan_analytic(t, R)
    ms = np.full(len(cands), np.nan)
    for c, cand in enumerate(cands):
        if nbytes[c] >= 90e9:
            continue
        plan = {"nmodes": cand["nmodes"], "groups": cand["groups"]}
        ms[c] = time_plan(t, plan, sweeps, R)
    return X, nbytes, cands, ms, chosen


def _save(path, rows, labels, tid, cidx, analytic, specs):
    np.savez(path, X=np.array(rows, dtype=np.float32).reshape(-1, A.PLAN_FEATURES),
             y=np.array(labels, dtype=np.float32), tensor=np.array(tid, dtype=np.int64),
             cand=np.array(cidx, dtype=np.int64), analytic=np.array(analytic, dtype=np.int64),
             specs=np.array(specs))


def make(args):
    import time
    A.lib().adatm_set_device(0)
    rows, labels, tid, cidx, analytic, specs = [], [], [], [], [], []
    ranks = [int(r) for r in args.ranks.split(",")]
    t_start = time.time()
    for k in range(args.tensors):
        if args.time_limit and time.time() - t_start > args.time_limit:
            print(f"time limit reached after {k} tensors", flush=True)
            break
        if k and args.checkpoint and k % args.checkpoint == 0:
            _save(args.out, rows, labels, tid, cidx, analytic, specs)
        seed = args.seed0 + k
        N, dims, nnz, alpha, R = draw_tensor_spec(seed, args.max_nnz, args.min_nnz, args.min_order,
                                                  ranks)
        t = A.Tensor.generate(dims, nnz, alpha=alpha, seed=seed)
        X, nbytes, cands, ms, chosen = measure_tensor(t, args.sweeps, R)
        t.free()
        for c in range(len(cands)):
            if np.isfinite(ms[c]):
                rows.append(X[c])
                labels.append(math.log10(ms[c]))
                tid.append(k)
                cidx.append(c)
        analytic.append(chosen)
        specs.append(json.dumps({"seed": seed, "N": N, "dims": dims, "nnz": nnz, "alpha": alpha,
                                 "R": R}))
        print(f"tensor {k} N={N} R={R} nnz={nnz} cands={len(cands)} ms={np.round(ms, 3).tolist()} "
              f"analytic={chosen}", flush=True)
    _save(args.out, rows, labels, tid, cidx, analytic, specs)


def regrets(y, tensor, cand, analytic, pred, ids):
    """Mean / max regret of the model's and the analytic choice over tensors
    `ids` (labels are log10 ms)."""
    out = {"learned": [], "analytic": []}
    for k in ids:
        m = tensor == k
        if not m.any():
            continue
        ms = 10.0 ** y[m]
        best = ms.min()
        out["learned"].append(ms[np.argmin(pred[m])] / best - 1.0)
        a = np.where(cand[m] == analytic[k])[0]
        out["analytic"].append((ms[a[0]] if len(a) else ms.max()) / best - 1.0)
    return {k: {"mean": float(np.mean(v)), "max": float(np.max(v)), "n": len(v)}
            for k, v in out.items()}


def load_sets(paths):
    """Union of data sets; tensor ids offset per set. Returns the arrays and
    a held-out mask per tensor (the last 20% of every set)."""
    Xs, ys, ts, cs, an, held = [], [], [], [], [], []
    off = 0
    for p in paths:
        z = np.load(p)
        nt = len(z["analytic"])
        split = int(round(nt * 0.8))
        Xs.append(z["X"])
        ys.append(z["y"])
        ts.append(z["tensor"] + off)
        cs.append(z["cand"])
        an.append(z["analytic"])
        held += [k >= split for k in range(nt)]
        off += nt
    return (np.concatenate(Xs), np.concatenate(ys), np.concatenate(ts), np.concatenate(cs),
            np.concatenate(an), np.array(held))


def train(args):
    A.lib().adatm_set_device(0)
    X, y, tensor, cand, analytic, held_t = load_sets(args.data)
    nt = len(analytic)
    tr = ~held_t[tensor]
    mean = X[tr].mean(axis=0)
    std = X[tr].std(axis=0)
    std[std < 1e-6] = 1.0
    Xs = (X - mean) / std
    net = A.Mlp(WIDTHS, seed=args.seed)
    loss = net.train(Xs[tr], y[tr], epochs=args.epochs, batch=args.batch, lr=args.lr, seed=args.seed)
    model = A.PlanModel(WIDTHS, net.get_params(), mean, std)
    pred = model.predict(X)
    held = [k for k in range(nt) if held_t[k]]
    rg = regrets(y, tensor, cand, analytic, pred, held)
    rg_train = regrets(y, tensor, cand, analytic, pred, [k for k in range(nt) if not held_t[k]])
    report = {"train_loss": loss, "rows": int(len(y)), "tensors": nt, "held_out_tensors": len(held),
              "held_out": rg, "train": rg_train, "data": [os.path.basename(p) for p in args.data]}
    model.save(args.model, report=json.dumps(report), held=held_t)
    print(json.dumps(report, indent=1))


BIG_DIMS = [50000, 20000, 10000, 2000, 500, 100]
BIG_NNZ = 100_000_000
BIG_ALPHA = 1.3


def evaluate(args):
    A.lib().adatm_set_device(0)
    model = A.PlanModel.load(args.model)
    if args.big:
        t = A.Tensor.generate(BIG_DIMS, BIG_NNZ, alpha=BIG_ALPHA, seed=args.big_seed)
    else:
        N, dims, nnz, alpha, _ = draw_tensor_spec(args.seed, args.max_nnz)
        t = A.Tensor.generate(dims, nnz, alpha=alpha, seed=args.seed)
    X, nbytes, cands, ms, chosen = measure_tensor(t, args.sweeps)
    _, learned, used = A.plan_learned(t, RANK, model)
    best = int(np.nanargmin(ms))
    out = {"tensor": {"dims": t.info()[2], "nnz": t.info()[1]},
           "ms_per_candidate": [None if not np.isfinite(v) else float(v) for v in ms],
           "best": best, "analytic": int(chosen), "learned": int(learned), "model_used": used,
           "regret_analytic": float(ms[chosen] / ms[best] - 1.0),
           "regret_learned": float(ms[learned] / ms[best] - 1.0),
           "predicted_log10_ms": model.predict(X).tolist()}
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    m = sub.add_parser("make")
    m.add_argument("--tensors", type=int, default=400)
    m.add_argument("--seed0", type=int, default=1000)
    m.add_argument("--max-nnz", type=float, default=4e6)
    m.add_argument("--min-nnz", type=float, default=1e5)
    m.add_argument("--min-order", type=int, default=4)
    m.add_argument("--ranks", default=str(RANK))
    m.add_argument("--sweeps", type=int, default=5)
    m.add_argument("--out", required=True)
    m.add_argument("--time-limit", type=float, default=0, help="stop after this many seconds")
    m.add_argument("--checkpoint", type=int, default=100, help="save every this many tensors")
    t = sub.add_parser("train")
    t.add_argument("--data", action="append", required=True)
    t.add_argument("--model", default=DEFAULT_MODEL)
    t.add_argument("--epochs", type=int, default=400)
    t.add_argument("--batch", type=int, default=128)
    t.add_argument("--lr", type=float, default=2e-3)
    t.add_argument("--seed", type=int, default=0)
    e = sub.add_parser("eval")
    e.add_argument("--model", default=DEFAULT_MODEL)
    e.add_argument("--big", action="store_true")
    e.add_argument("--big-seed", type=int, default=0, help="seed of the held-out 6th-order tensor")
    e.add_argument("--seed", type=int, default=99999)
    e.add_argument("--max-nnz", type=float, default=4e6)
    e.add_argument("--sweeps", type=int, default=5)
    a = ap.parse_args()
    {"make": make, "train": train, "eval": evaluate}[a.cmd](a)


if __name__ == "__main__":
    sys.exit(main())
