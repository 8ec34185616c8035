"""Run CP-ALS sweeps on a seeded synthetic tensor (for profilers).

    python -m adatm_b200.profile_case [--nnz 8000000] [--sweeps 3] [--dims 5000,5000,2000,500]
                                      [--alpha 1.1] [--rank 32] [--bf16] [--plain] [--lognormal]
                                      [--groups JSON] [--walkers W] [--fold F] [--atomic] [--time]

Builds the tensor, the analytic plan (the plain one-tree-per-mode plan with
--plain, or the given group list) and the engine on device 0, then runs the given number of sweeps
without a CUDA graph, so a profiler sees each kernel launch.
"""
import argparse
import json

import adatm_b200 as A


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nnz", type=int, default=8_000_000)
    ap.add_argument("--dims", default="5000,5000,2000,500")
    ap.add_argument("--alpha", type=float, default=1.1)
    ap.add_argument("--rank", type=int, default=32)
    ap.add_argument("--sweeps", type=int, default=3)
    ap.add_argument("--bf16", action="store_true")
    ap.add_argument("--plain", action="store_true")
    ap.add_argument("--time", action="store_true", help="print per-mode MTTKRP and sweep times")
    ap.add_argument("--chunk", type=int, default=0, help="source units per chunk (0 = default)")
    ap.add_argument("--lognormal", action="store_true", help="values lognormal(0, 1) instead of U(0, 1)")
    ap.add_argument("--groups", default=None,
                    help="the plan's group list as JSON (memo_mode, begin_imten, n_imten, o_opt "
                         "per group) instead of the analytic plan")
    ap.add_argument("--walkers", type=int, default=0, help="walkers per warp (0 = default)")
    ap.add_argument("--fold", type=int, default=-1, help="levels folded into the source loop (-1 = chosen)")
    ap.add_argument("--atomic", action="store_true", help="atomic scatters (not deterministic)")
    a = ap.parse_args()
    dims = [int(x) for x in a.dims.split(",")]
    A.lib().adatm_set_device(0)
    t = A.Tensor.generate(dims, a.nnz, alpha=a.alpha, value_kind=1 if a.lognormal else 0, seed=0)
    if a.plain:
        plan = A.plan_splatt(t, A.CSF_ALLMODE)
    elif a.groups:
        plan = {"nmodes": len(dims), "groups": json.loads(a.groups)}
    else:
        plan = A.plan_analytic(t, a.rank)[0]
    e = A.Engine(t, a.rank, plan, bf16=a.bf16, chunk_leaf=a.chunk, chunk_rows=a.chunk)
    if a.walkers:
        e.set_walkers(a.walkers)
    if a.fold != -1:
        e.set_fold(a.fold)
    if a.atomic:
        e.set_deterministic(False)
    e.init_factors(0)
    res = e.als(a.sweeps, 0.0, graph=False)
    print(f"nnz {t.info()[1]} plan {plan['groups']} fit {res['fit']:.6f} trace {res['trace']}")
    if a.time:
        n = len(dims)
        tags = plan.get("use_tags") or A.decide_use_csfs(n, plan["groups"])[1]
        for m in range(n):
            e.time_mttkrp(m, 3)
            ms = e.time_mttkrp(m, 20) / 20
            gbs = e.mttkrp_bytes(m) / (ms * 1e-3) / 1e9
            print(f"mode {m} tag {tags[m]}: {ms * 1e3:8.1f} us  {gbs:7.1f} GB/s compulsory")
        e.als_begin(graph=True)
        e.time_sweeps(3)
        print(f"sweep (graph): {e.time_sweeps(50) / 50:.3f} ms")


if __name__ == "__main__":
    main()
