"""CP-ALS sweep benchmark on the AdaTM memoized MTTKRP path (B200).

One step = one CP-ALS sweep (iteration): N MTTKRPs following the memo plan,
N dense mode updates (FP64 Gram Hadamard + inverse, FP32 rows) and the fit.
The default workload is the largest single-GPU configuration, the held-out
6th-order tensor 50000 x 20000 x 10000 x 2000 x 500 x 100 with 100M Zipf(1.3)
draws (duplicates summed), values uniform(0,1), rank 32, FP32, on the plan
the learned plan model picks. A second section measures the 5th-order BF16
workload (20000 x 10000 x 5000 x 1000 x 200, 50M Zipf(1.2) draws, lognormal
values, rank 64) with each mode's MTTKRP error and the fit against FP64.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload held_out_6mode|bf16_5mode|zipf_4mode|uniform_3mode]

Prints one JSON line. --impl reference times the reference's own CPU code
(oracle/_ref: the reference's AdaTM C files; else the oracle restatement) on
the host cores, on a bounded random sample of the same workload's nonzeros
(the time scaled to the whole tensor), without loading this library: the
tensor comes from the host port of the seeded generator. With --gpus N > 1
(torchrun) every rank runs an independent replica ("replicas only"); the time
is the maximum over ranks.
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
SEED = 0
FALLBACK_HBM = 6650.0

WORKLOADS = {
    "held_out_6mode": {
        "dims": [50000, 20000, 10000, 2000, 500, 100], "nnz_drawn": 100_000_000, "alpha": 1.3,
        "values": "uniform(0,1)", "value_kind": 0, "rank": 32, "precision": "fp32", "iters": 20,
        "text": "6th-order 50000x20000x10000x2000x500x100, 100M Zipf(1.3) draws per mode "
                "(duplicates summed), values U(0,1), R=32, FP32, learned memo plan, one CP-ALS "
                "sweep per step"},
    "bf16_5mode": {
        "dims": [20000, 10000, 5000, 1000, 200], "nnz_drawn": 50_000_000, "alpha": 1.2,
        "values": "lognormal(0,1)", "value_kind": 1, "rank": 64, "precision": "bf16", "iters": 10,
        "text": "5th-order 20000x10000x5000x1000x200, 50M Zipf(1.2) draws per mode (duplicates "
                "summed), values lognormal(0,1), R=64, BF16 factor rows with FP32 accumulation, "
                "one CP-ALS sweep per step"},
    "zipf_4mode": {
        "dims": [5000, 5000, 2000, 500], "nnz_drawn": 20_000_000, "alpha": 1.1,
        "values": "uniform(0,1)", "value_kind": 0, "rank": 32, "precision": "fp32", "iters": 20,
        "text": "4th-order 5000x5000x2000x500, 20M Zipf(1.1) draws per mode (duplicates summed), "
                "values U(0,1), R=32, FP32, memoized plan, one CP-ALS sweep per step"},
    "uniform_3mode": {
        "dims": [1000, 1000, 1000], "nnz_drawn": 1_000_000, "alpha": None,
        "values": "uniform(0,1)", "value_kind": 0, "rank": 16, "precision": "fp32", "iters": 10,
        "text": "3rd-order 1000x1000x1000, 1M uniform draws (duplicates summed), values U(0,1), "
                "R=16, FP32, one CP-ALS sweep per step"},
}
HEADLINE = "held_out_6mode"
SECOND = "bf16_5mode"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def config_of(name):
    """The `config` object both arms print for a workload (static, so the two
    lines carry the same dict)."""
    w = WORKLOADS[name]
    return {"workload": w["text"], "dims": w["dims"], "nnz_drawn": w["nnz_drawn"],
            "zipf_alpha": w["alpha"], "values": w["values"], "rank": w["rank"],
            "precision": w["precision"], "seed": SEED,
            "l2": "inputs larger than L2 (trees and memo rows of several GB streamed every sweep)",
            "parallelism": "single GPU per rank (replicas for N > 1)"}


def peaks():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM, "fallback"


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


def sample_nonzeros(inds, vals, fraction, seed=SEED):
    """A seeded random subset (about `fraction`) of the nonzeros, dims kept:
    the bounded sample the CPU timings run on."""
    if fraction >= 1.0:
        return inds, vals
    rng = np.random.default_rng(seed + 12345)
    keep = rng.random(len(vals)) < fraction
    return np.ascontiguousarray(inds[:, keep]), np.ascontiguousarray(vals[keep])


class ReferenceRun:
    """The reference's own CPU code (or the oracle port) on a bounded sample
    of a workload: its planner, csf_alloc_adaptive / rcsf_alloc_adaptive and
    cpd_als_iterate_adaptive sweeps."""

    def __init__(self, inds, vals, dims, rank, fraction, nthreads):
        import oracle as O
        self.O = O
        self.kind = "reference" if O.ref_available() else "port"
        sinds, svals = sample_nonzeros(inds, vals, fraction)
        self.fraction = len(svals) / max(1, len(vals))
        self.nnz = len(svals)
        self.threads = nthreads
        t0 = time.perf_counter()
        groups = O.ref_plan(sinds, svals, dims, rank) if self.kind == "reference" else None
        if groups is None:  # the oracle port, or N == 3 where the reference's planner is undefined
            groups, _ = O.plan(sinds, dims, rank)
        if self.kind == "reference":
            self.model = O.RefModel(sinds, svals, dims, rank, groups, nthreads=nthreads)
        else:
            self.model = O.Model(sinds, svals, dims, rank, groups)
        self.groups = groups
        self.setup_s = time.perf_counter() - t0
        self.mats = O.init_factors(dims, rank, SEED)

    def sweeps_s(self, n):
        """Seconds for n CP-ALS sweeps of the sample (one call)."""
        t0 = time.perf_counter()
        if self.kind == "reference":
            self.model.cpd_als(self.mats, n, 0.0, zero_memo=False)
        else:
            self.model.cpd_als(self.mats, n, 0.0)
        return time.perf_counter() - t0

    def ms_per_sweep_scaled(self, seconds, n):
        """Sample time per sweep scaled to the whole tensor by its nonzeros."""
        return 1e3 * seconds / n / self.fraction

    def describe(self, n):
        src = (f"the reference's AdaTM C files (-O3 -march={self.O.ref_build_arch()})"
               if self.kind == "reference" else "the oracle port")
        return (f"{n} CP-ALS sweeps of {src} (FP64, {self.threads} OpenMP threads) on a seeded "
                f"random {self.fraction:.4f} of the nonzeros ({self.nnz} of them, same dims), "
                f"time per sweep scaled by 1/{self.fraction:.4f}")


def reference_fraction(name):
    """Sample size of the CPU timings: a few million nonzeros."""
    w = WORKLOADS[name]
    return min(1.0, 4_000_000 / w["nnz_drawn"])


def run_reference(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    import oracle as O  # the host generator port: this arm never loads the GPU library
    name = args.workload
    w = WORKLOADS[name]
    threads = host_threads(int(4_000_000 * w["rank"] * 8 * 1.5))
    O.threads(threads)
    t0 = time.perf_counter()
    inds, vals, dims = O.generate(w["dims"], w["nnz_drawn"], alpha=w["alpha"],
                                  value_kind=w["value_kind"], seed=SEED)
    gen_s = time.perf_counter() - t0
    ref = ReferenceRun(inds, vals, dims, w["rank"], reference_fraction(name), threads)
    del inds, vals
    W, K = max(0, args.warmup), max(1, args.steps)
    if W:
        ref.sweeps_s(W)
    sec = ref.sweeps_s(K)
    ms = ref.ms_per_sweep_scaled(sec, K)
    line = {"metric": METRIC, "value": ms, "unit": "ms/sweep", "n_gpus": args.gpus,
            "steps": K, "warmup": W, "ms_per_step": ms,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded host generator with the workload's shapes and distributions)",
            "config": config_of(name),
            "impl": "reference",
            "cpu_baseline": {"value": ms, "unit": "ms/sweep", "cores": threads, "kind": ref.kind,
                             "sample": ref.describe(K)},
            "e2e": {"value": ms, "unit": "ms/sweep", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "setup_s": {"generate": gen_s, "plan_and_build_sample": ref.setup_s}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def generate_on_device(A, name):
    w = WORKLOADS[name]
    return A.Tensor.generate(w["dims"], w["nnz_drawn"], alpha=w["alpha"], value_kind=w["value_kind"],
                             seed=SEED)


def time_engine(A, t, rank, plan, W, K, bf16=False):
    e = A.Engine(t, rank, plan, bf16=bf16)
    e.init_factors(SEED)
    e.als_begin(graph=True)
    e.time_sweeps(W)
    ms = e.time_sweeps(K) / K
    e.free()
    return ms


def start_factors32(O, dims, rank):
    """The seeded start factors as the device holds them (FP32-rounded), in
    FP64, so the FP64 oracle starts from exactly the GPU's start."""
    return [np.asarray(m, dtype=np.float32).astype(np.float64) for m in O.init_factors(dims, rank, SEED)]


def fit_check(A, O, t, rank, plan, inds, vals, dims, iters, bf16=False):
    """Fit trace of `iters` sweeps on the GPU and of the FP64 oracle (COO
    MTTKRP, the reference's ALS steps) from the same start factors."""
    g = A.Engine(t, rank, plan, bf16=bf16)
    g.init_factors(SEED)
    r = g.als(iters, 0.0, graph=True)
    g.free()
    t0 = time.perf_counter()
    ref = O.cpd_als_coo(inds, vals, dims, rank, start_factors32(O, dims, rank), iters, 0.0)
    return {"sweeps": iters, "fit_gpu": r["fit"], "fit_fp64": ref["fit"],
            "delta": abs(r["fit"] - ref["fit"]),
            "max_delta_over_sweeps": float(np.max(np.abs(np.array(r["trace"]) - ref["trace"]))),
            "fp64_s": time.perf_counter() - t0}


def mttkrp_errors(A, O, t, rank, plan, inds, vals, dims, bf16):
    """Relative Frobenius error of every mode's MTTKRP (the plan's sequence:
    memo root, then the reuse modes) against the FP64 oracle, from the
    seeded start factors."""
    e = A.Engine(t, rank, plan, bf16=bf16)
    start = start_factors32(O, dims, rank)
    e.set_factors(start)
    out = []
    for m in range(len(dims)):
        got = e.mttkrp(m)
        want = O.mttkrp_coo(inds, vals, dims, start, m, rank)
        out.append(float(np.linalg.norm(got - want) / np.linalg.norm(want)))
    e.free()
    return out


def load_model(A):
    path = os.path.join(HERE, "adatm_b200", "planner_data", "plan_model.npz")
    return A.PlanModel.load(path) if os.path.exists(path) else None


def second_section(A, O, W, K):
    """The 5th-order BF16 workload: BF16 and FP32 sweeps, the plain rCSF
    sweep, each mode's MTTKRP error and the fit after its sweeps vs FP64."""
    w = WORKLOADS[SECOND]
    t = generate_on_device(A, SECOND)
    _, nnz, dims = t.info()
    inds, vals, _ = t.download()
    plan, idx, used = A.plan_learned(t, w["rank"], load_model(A))
    res = {"workload": w["text"], "nnz": nnz, "plan": plan["groups"], "use_tags": plan["use_tags"],
           "bf16_sweep_ms": time_engine(A, t, w["rank"], plan, W, K, bf16=True),
           "fp32_sweep_ms": time_engine(A, t, w["rank"], plan, W, K),
           "plain_rcsf_fp32_sweep_ms": time_engine(A, t, w["rank"], A.plan_splatt(t, A.CSF_ALLMODE),
                                                   W, K),
           "mttkrp_relerr_bf16": mttkrp_errors(A, O, t, w["rank"], plan, inds, vals, dims, True),
           "mttkrp_relerr_fp32": mttkrp_errors(A, O, t, w["rank"], plan, inds, vals, dims, False),
           "fit_check_bf16": fit_check(A, O, t, w["rank"], plan, inds, vals, dims, w["iters"], True),
           "fit_check_fp32": fit_check(A, O, t, w["rank"], plan, inds, vals, dims, w["iters"], False)}
    t.free()
    return res


def run_ours(args):
    world, rank, local = dist_setup()
    import adatm_b200 as A
    A.lib()
    if A.lib().adatm_set_device(local) != A.SPLATT_SUCCESS:
        raise RuntimeError(A._native.last_error())
    name = args.workload
    w = WORKLOADS[name]
    R = w["rank"]
    bf16 = w["precision"] == "bf16"
    t0 = time.perf_counter()
    t = generate_on_device(A, name)
    nmodes, nnz, dims = t.info()
    gen_s = time.perf_counter() - t0
    # the chosen plan: the learned plan model shipped with the package (the
    # analytic model when it is absent); the analytic plan is timed beside it
    t0 = time.perf_counter()
    plan, chosen_idx, model_used = A.plan_learned(t, R, load_model(A))
    plan_s = time.perf_counter() - t0
    analytic_plan, cands, analytic_idx = A.plan_analytic(t, R)
    t0 = time.perf_counter()
    eng = A.Engine(t, R, plan, bf16=bf16)
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

    # dominant kernel: the slowest MTTKRP of the sweep
    reps = 10
    mode_ms = []
    for m in range(nmodes):
        eng.time_mttkrp(m, 3)
        mode_ms.append(eng.time_mttkrp(m, reps) / reps)
    dom = int(np.argmax(mode_ms))
    dom_bytes = eng.mttkrp_bytes(dom)
    achieved = dom_bytes / (mode_ms[dom] * 1e-3) / 1e9
    peak, peak_kind = peaks()
    bytes_per_mode = [eng.mttkrp_bytes(m) for m in range(nmodes)]
    seq_gbs = sum(bytes_per_mode) / (sum(mode_ms) * 1e-3) / 1e9
    eng.free()

    # plain GPU rCSF (one tree per mode, no memo), every candidate plan
    # (exhaustive search) and the other precision, same GPU
    plain_ms = time_engine(A, t, R, A.plan_splatt(t, A.CSF_ALLMODE), W, K, bf16=bf16)
    cand_ms = []
    if rank == 0 and not args.quick:
        for c in cands:
            cplan = {k: c[k] for k in ("nmodes", "groups", "use_csfs", "use_tags", "space_efficient")}
            cand_ms.append(time_engine(A, t, R, cplan, 2, max(3, K // 4), bf16=bf16))
    other_ms = time_engine(A, t, R, plan, W, K, bf16=not bf16)

    # end to end through the drop-in C ABI with host buffers:
    # cpd_als_iterate_adaptive(NITER=1) per step (factors in, factors out)
    inds, vals, _ = t.download()
    groups = plan["groups"]
    cs = A.csf_alloc_adaptive(inds, vals, dims, groups)
    rs = A.rcsf_alloc_adaptive(cs, R, groups)
    uc, ut = A.decide_use_csfs(nmodes, groups, len(cs))
    rng = np.random.default_rng(SEED)
    mats = [rng.random((d, R)) for d in dims]
    it = A.CpdIterator(cs, rs, groups, uc, ut, mats)
    it.step(1)
    E = max(3, min(K, 20))
    barrier(world)
    te = time.perf_counter()
    for _ in range(E):
        it.step(1)  # factors in and out of the same host buffers
    e2e_s = max_over_ranks(time.perf_counter() - te, world)
    ldr = (R + 3) // 4 * 4
    h2d = sum(dims) * ldr * 4
    d2h = sum(dims) * ldr * 4 + R * 8 + 8
    cs.free()

    # rank 0: the fit after the workload's sweeps against the FP64 oracle, the
    # reference CPU baseline on a bounded sample, and the second workload
    cpu = fitc = second = None
    if rank == 0 and not args.no_cpu:
        import oracle as O
        threads = host_threads(int(4_000_000 * R * 8 * 1.5))
        O.threads(threads)
        fitc = fit_check(A, O, t, R, plan, inds, vals, dims, w["iters"], bf16)
        ref = ReferenceRun(inds, vals, dims, R, reference_fraction(name), threads)
        ref.sweeps_s(1)
        n = 3
        cpu = {"value": ref.ms_per_sweep_scaled(ref.sweeps_s(n), n), "unit": "ms/sweep",
               "cores": threads, "kind": ref.kind, "sample": ref.describe(n)}
        del ref
        if not args.quick and name == HEADLINE:
            del inds, vals
            t.free()
            second = second_section(A, O, W, K)
    t.free()

    if rank != 0:
        return 0
    cand_info = None
    if cand_ms:
        best = int(np.argmin(cand_ms))
        cand_info = {"ms_per_sweep": cand_ms, "best": best, "learned_choice": chosen_idx,
                     "analytic_choice": analytic_idx,
                     "learned_regret": cand_ms[chosen_idx] / cand_ms[best] - 1,
                     "analytic_regret": cand_ms[analytic_idx] / cand_ms[best] - 1}
    line = {
        "metric": METRIC, "value": replica_ms_per_sweep(ms_total, K, world), "unit": "ms/sweep",
        "n_gpus": world,
        "steps": K, "warmup": W, "ms_per_step": ms_step, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16" if bf16 else "f32",
        "data": "synthetic (seeded device generator with the workload's shapes and distributions)",
        "config": config_of(name),
        "workload_detail": {"nnz": nnz, "dims": dims, "plan": plan["groups"],
                            "use_tags": plan["use_tags"],
                            "device_bytes": {"trees": csf_b, "memo_rows": memo_b},
                            "graph": "one sweep captured in a CUDA graph"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "peak_source": peak_kind,
                     "kernel": f"MTTKRP mode {dom} (tag {plan['use_tags'][dom]})",
                     "algorithmic_bytes_per_launch": dom_bytes},
        "gpu_launches": per_sweep * K,
        "clocks": clk,
        "e2e": {"value": 1e3 * e2e_s / E, "unit": "ms/sweep", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "call": "cpd_als_iterate_adaptive(NITER=1) with host FP64 factors per step"},
        "chosen_vs_plain": {"chosen_sweep_ms": ms_step,
                            ("fp32" if bf16 else "bf16") + "_sweep_ms": other_ms,
                            "plain_rcsf_sweep_ms": plain_ms,
                            "speedup_chosen_vs_plain": plain_ms / ms_step,
                            "plan_model": "learned" if model_used else "analytic",
                            "chosen_candidate": chosen_idx, "analytic_candidate": analytic_idx},
        "plan_search": cand_info,
        "mttkrp": {"ms_per_mode": mode_ms, "sequence_gbs": seq_gbs, "bytes_per_mode": bytes_per_mode},
        "fit_check": fitc,
        "setup_s": {"generate": gen_s, "plan": plan_s, "build": build_s},
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if second is not None:
        line[SECOND] = second
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default=HEADLINE)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU legs (oracle fit, baseline)")
    ap.add_argument("--quick", action="store_true", help="skip the plan search and second workload")
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
