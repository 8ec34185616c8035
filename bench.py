"""CP-ALS sweep benchmark on the AdaTM memoized MTTKRP path (B200).

One step = one CP-ALS sweep (iteration): N MTTKRPs following the memo plan,
N dense mode updates (FP64 Gram Hadamard + Cholesky inverse, FP32 rows) and
the fit, over the 4th-order workload 5000 x 5000 x 2000 x 500 with 20M
Zipf(1.1) draws (duplicates summed), values uniform(0,1), rank 32, FP32,
generated on the device from seed 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line. --impl reference times the reference's own CPU code
(oracle/_ref, the reference's AdaTM C files; else the oracle restatement) on
the host cores for the same workload. With --gpus N > 1 (torchrun) every rank
runs an independent replica ("replicas only": one tensor does not shard in
this path); the time is the maximum over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "CP-ALS sweep ms + MTTKRP HBM GB/s, chosen vs plain GPU rCSF at fit Δ≤1e-4"
DIMS = [5000, 5000, 2000, 500]
NNZ_DRAWN = 20_000_000
ALPHA = 1.1
RANK = 32
SEED = 0
WORKLOAD = ("4th-order 5000x5000x2000x500, 20M Zipf(1.1) draws per mode (duplicates summed), "
            "values U(0,1), R=32, FP32, memoized AdaTM plan, one CP-ALS sweep per step")
FALLBACK_HBM = 6650.0


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def peaks():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM, "fallback"


def profiled_traffic(mode):
    """Per-launch DRAM bytes of mode `mode`'s MTTKRP from the committed ncu
    summary (profiles/mttkrp_walk.md, line 'traffic_bytes_per_launch[mode M]: X')."""
    p = os.path.join(HERE, "profiles", "mttkrp_walk.md")
    if not os.path.exists(p):
        return None
    key = f"traffic_bytes_per_launch[mode {mode}]:"
    for line in open(p):
        if line.strip().startswith(key):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


class Clocks:
    """nvidia-smi samples during the timed region."""

    Q = ("index,pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id=None):
        self.bus_id = bus_id
        self.proc = None
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.file.read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 10:
                continue
            if self.bus_id and self.bus_id.lower() not in parts[1].lower():
                continue
            try:
                sm.append(float(parts[2]))
                smax = float(parts[3])
            except ValueError:
                continue
            for n, v in zip(names, parts[6:10]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.file.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(backend=None):
    """One process per GPU from torchrun's environment. The backend is NCCL
    when CUDA is present (gloo otherwise, which the CPU tests use)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def max_over_ranks(x, world):
    """Maximum of a per-rank scalar (the device time of the timed region)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def replica_ms_per_sweep(ms_total_max, steps, world):
    """Whole-job ms per sweep for `world` independent replicas that each ran
    `steps` sweeps in ms_total_max (the slowest rank's time)."""
    return ms_total_max / (steps * world)


# ---------------------------------------------------------------------------
# reference CPU code (oracle/_ref) on the host cores
# ---------------------------------------------------------------------------

def host_threads(tmp_bytes_per_thread):
    ncpu = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    avail = None
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable:"):
                avail = int(line.split()[1]) * 1024
    except OSError:
        pass
    if avail and tmp_bytes_per_thread > 0:
        ncpu = max(1, min(ncpu, int(0.4 * avail // tmp_bytes_per_thread)))
    return ncpu


def reference_sweeps(inds, vals, dims, nsweeps, budget_s, nthreads, zero_memo, seed=SEED):
    """Time up to nsweeps CP-ALS sweeps of the reference (or the oracle port)
    within budget_s seconds. Returns dict with per-sweep ms and the fit."""
    import oracle as O
    kind = "reference" if O.ref_available() else "port"
    t0 = time.perf_counter()
    if kind == "reference":
        groups = O.ref_plan(inds, vals, dims, RANK)
        model = O.RefModel(inds, vals, dims, RANK, groups, nthreads=nthreads)
    else:
        groups, _ = O.plan(inds, dims, RANK)
        model = O.Model(inds, vals, dims, RANK, groups)
    build_s = time.perf_counter() - t0
    mats = O.init_factors(dims, RANK, seed)
    # one sweep to size the sample, then as many as fit the budget
    t1 = time.perf_counter()
    if kind == "reference":
        res = model.cpd_als(mats, 1, 0.0, zero_memo=zero_memo)
    else:
        res = model.cpd_als(mats, 1, 0.0)
    one = time.perf_counter() - t1
    n = int(max(1, min(nsweeps, budget_s // max(one, 1e-3))))
    t2 = time.perf_counter()
    if kind == "reference":
        res = model.cpd_als(mats, n, 0.0, zero_memo=zero_memo)
    else:
        res = model.cpd_als(mats, n, 0.0)
    el = time.perf_counter() - t2
    return {"kind": kind, "ms_per_sweep": 1e3 * el / n, "sweeps": n, "fit": res["fit"],
            "build_s": build_s, "groups": groups}


def generate_workload(A):
    t = A.Tensor.generate(DIMS, NNZ_DRAWN, alpha=ALPHA, value_kind=0, seed=SEED)
    return t


def run_reference(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    import adatm_b200 as A
    A.lib()
    A.lib().adatm_set_device(local)
    # the device only synthesises the input tensor (untimed); the timed path
    # is the reference's own CPU code
    t = generate_workload(A)
    inds, vals, dims = t.download()
    t.free()
    plan_nf = 4 * (int(max(dims)) * 64) * RANK * 8
    threads = host_threads(int(len(vals) * RANK * 8 * 1.5) or plan_nf)
    budget = 150.0
    res = reference_sweeps(inds, vals, dims, max(1, args.steps), budget, threads, zero_memo=False)
    line = {"metric": METRIC, "value": res["ms_per_sweep"], "unit": "ms/sweep", "n_gpus": args.gpus,
            "steps": res["sweeps"], "warmup": 1, "ms_per_step": res["ms_per_sweep"],
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator, the workload's shapes and distributions)",
            "config": {"workload": WORKLOAD, "dims": dims, "nnz": int(len(vals)), "rank": RANK},
            "impl": "reference",
            "cpu_baseline": {"value": res["ms_per_sweep"], "unit": "ms/sweep", "cores": threads,
                             "kind": res["kind"],
                             "sample": f"{res['sweeps']} full CP-ALS sweeps of the workload "
                                       f"({'reference AdaTM C files' if res['kind'] == 'reference' else 'oracle port'}, "
                                       f"{threads} OpenMP threads, FP64)"},
            "e2e": {"value": res["ms_per_sweep"], "unit": "ms/sweep", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def run_ours(args):
    world, rank, local = dist_setup()
    import adatm_b200 as A
    A.lib()
    if A.lib().adatm_set_device(local) != A.SPLATT_SUCCESS:
        raise RuntimeError(A._native.last_error())
    t0 = time.perf_counter()
    t = generate_workload(A)
    nmodes, nnz, dims = t.info()
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    # the chosen plan: the learned plan model shipped with the package (the
    # analytic model when it is absent); the analytic plan is timed beside it
    model_path = os.path.join(HERE, "adatm_b200", "planner_data", "plan_model.npz")
    model = A.PlanModel.load(model_path) if os.path.exists(model_path) else None
    plan, chosen_idx, model_used = A.plan_learned(t, RANK, model)
    plan_s = time.perf_counter() - t0
    analytic_plan, _, analytic_idx = A.plan_analytic(t, RANK)
    t0 = time.perf_counter()
    eng = A.Engine(t, RANK, plan)
    build_s = time.perf_counter() - t0
    csf_b, memo_b = eng.memory()
    eng.init_factors(SEED)
    eng.als_begin(graph=True)
    per_sweep, _ = eng.launch_counts(0)
    W = max(3, args.warmup)
    K = max(1, args.steps)
    eng.time_sweeps(W)
    bus = None
    try:
        import torch
        p = torch.cuda.get_device_properties(local)
        bus = getattr(p, "pci_bus_id", None)
        if bus is not None:
            bus = f"{getattr(p, 'pci_domain_id', 0):08X}:{bus:02X}:{getattr(p, 'pci_device_id', 0):02X}"
    except Exception:
        bus = None
    clocks = Clocks(bus)
    barrier(world)
    clocks.start()
    time.sleep(0.1)
    ms_total = eng.time_sweeps(K)
    clk = clocks.stop()
    barrier(world)
    ms_total = max_over_ranks(ms_total, world)
    ms_step = ms_total / K
    fit = eng.fit()

    # dominant kernel: the slowest MTTKRP of the sweep
    reps = 20
    mode_ms = []
    for m in range(nmodes):
        eng.time_mttkrp(m, 3)
        mode_ms.append(eng.time_mttkrp(m, reps) / reps)
    dom = int(np.argmax(mode_ms))
    dom_bytes = eng.mttkrp_bytes(dom)
    achieved = dom_bytes / (mode_ms[dom] * 1e-3) / 1e9
    peak, peak_kind = peaks()
    seq_bytes = sum(eng.mttkrp_bytes(m) for m in range(nmodes))
    seq_gbs = seq_bytes / (sum(mode_ms) * 1e-3) / 1e9
    traffic = profiled_traffic(dom)

    # plain GPU rCSF (one tree per mode, no memo) and BF16 gathers, same GPU
    plain = A.Engine(t, RANK, A.plan_splatt(t, A.CSF_ALLMODE))
    plain.init_factors(SEED)
    plain.als_begin(graph=True)
    plain.time_sweeps(W)
    plain_ms = plain.time_sweeps(K) / K
    plain.free()
    if analytic_idx != chosen_idx:
        an = A.Engine(t, RANK, analytic_plan)
        an.init_factors(SEED)
        an.als_begin(graph=True)
        an.time_sweeps(W)
        analytic_ms = an.time_sweeps(K) / K
        an.free()
    else:
        analytic_ms = None  # same plan as the chosen one
    bf = A.Engine(t, RANK, plan, bf16=True)
    bf.init_factors(SEED)
    bf.als_begin(graph=True)
    bf.time_sweeps(W)
    bf_ms = bf.time_sweeps(K) / K
    bf.free()

    # end to end through the drop-in C ABI with host buffers:
    # cpd_als_iterate_adaptive(NITER=1) per step (factors in, factors out)
    inds, vals, _ = t.download()
    groups = plan["groups"]
    cs = A.csf_alloc_adaptive(inds, vals, dims, groups)
    rs = A.rcsf_alloc_adaptive(cs, RANK, groups)
    uc, ut = A.decide_use_csfs(nmodes, groups, len(cs))
    rng = np.random.default_rng(SEED)
    mats = [rng.random((d, RANK)) for d in dims]
    it = A.CpdIterator(cs, rs, groups, uc, ut, mats)
    it.step(1)
    E = max(3, min(K, 20))
    barrier(world)
    te = time.perf_counter()
    for _ in range(E):
        it.step(1)  # factors in and out of the same host buffers
    e2e_s = max_over_ranks(time.perf_counter() - te, world)
    ldr = (RANK + 3) // 4 * 4
    h2d = sum(dims) * ldr * 4
    d2h = sum(dims) * ldr * 4 + RANK * 8 + 8
    cs.free()

    # reference CPU baseline on rank 0: a bounded sample of the same workload,
    # plus the fit after 2 sweeps against the GPU's from the same start
    cpu = None
    fit_check = None
    if rank == 0 and not args.no_cpu:
        threads = host_threads(int(nnz * RANK * 8 * 1.5))
        cpu = reference_sweeps(inds, vals, dims, 50, 20.0, threads, zero_memo=False)
        ref2 = reference_sweeps(inds, vals, dims, 2, 0.0, 1, zero_memo=True)
        g2 = A.Engine(t, RANK, plan)
        g2.init_factors(SEED)
        r2 = g2.als(ref2["sweeps"], 0.0, graph=False)
        fit_check = {"sweeps": ref2["sweeps"], "fit_gpu": r2["fit"], "fit_reference": ref2["fit"],
                     "delta": abs(r2["fit"] - ref2["fit"])}
        g2.free()

    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": replica_ms_per_sweep(ms_total, K, world), "unit": "ms/sweep",
        "n_gpus": world,
        "steps": K, "warmup": W, "ms_per_step": ms_step, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded device generator with the workload's shapes and distributions)",
        "config": {"workload": WORKLOAD, "dims": dims, "nnz_drawn": NNZ_DRAWN, "nnz": nnz,
                   "rank": RANK, "plan": plan["groups"], "use_tags": plan["use_tags"],
                   "parallelism": "replicas" if world > 1 else "single GPU",
                   "l2": f"inputs larger than L2: {(csf_b + memo_b) / 1e9:.2f} GB of trees and memo rows "
                         "resident and streamed every sweep",
                   "graph": "one sweep captured in a CUDA graph"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                     "kernel": f"MTTKRP mode {dom} (tag {plan['use_tags'][dom]})",
                     "algorithmic_bytes_per_launch": dom_bytes},
        "gpu_launches": per_sweep * K,
        "clocks": clk,
        "e2e": {"value": 1e3 * e2e_s / E, "unit": "ms/sweep", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "call": "cpd_als_iterate_adaptive(NITER=1) with host FP64 factors per step"},
        "chosen_vs_plain": {"memo_fp32_sweep_ms": ms_step, "memo_bf16_sweep_ms": bf_ms,
                            "plain_rcsf_fp32_sweep_ms": plain_ms,
                            "speedup_memo_vs_plain": plain_ms / ms_step,
                            "plan_model": "learned" if model_used else "analytic",
                            "chosen_candidate": chosen_idx, "analytic_candidate": analytic_idx,
                            "analytic_plan_sweep_ms": analytic_ms if analytic_ms is not None else ms_step},
        "mttkrp": {"ms_per_mode": mode_ms, "sequence_gbs": seq_gbs,
                   "bytes_per_mode": [eng.mttkrp_bytes(m) for m in range(nmodes)]},
        "fit_after_steps": fit,
        "fit_check": fit_check,
        "setup_s": {"generate": gen_s, "plan": plan_s, "build": build_s},
    }
    if cpu is not None:
        line["cpu_baseline"] = {"value": cpu["ms_per_sweep"], "unit": "ms/sweep", "cores": threads,
                                "kind": cpu["kind"],
                                "sample": f"{cpu['sweeps']} full CP-ALS sweeps of the same tensor "
                                          f"({cpu['kind']}, FP64, {threads} threads)"}
    print(json.dumps(line), flush=True)
    eng.free()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    args = ap.parse_args()
    if args.impl == "reference":
        rc = run_reference(args)
    else:
        rc = run_ours(args)
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()
    return rc


if __name__ == "__main__":
    sys.exit(main())
