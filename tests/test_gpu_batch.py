"""Batched sweeps of several uneven tensors in one CUDA graph, and the chunk
autotuner: both leave the numbers of a sweep unchanged."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [([300, 200, 100], 20000, None), ([120, 90, 80, 70], 30000, 1.2),
          ([60, 50, 40, 30, 20], 25000, 1.1), ([500, 40, 300], 15000, 1.4),
          ([90, 80, 70, 60], 5000, None), ([2000, 1500, 900], 60000, 1.3)]


def engines(A, R=16):
    out = []
    for k, (dims, nnz, alpha) in enumerate(SHAPES):
        t = A.Tensor.generate(dims, nnz, alpha=alpha, seed=100 + k)
        plan, _, _ = A.plan_analytic(t, R)
        out.append((t, A.Engine(t, R, plan)))
    return out


def test_batched_graph_matches_each_engine(gpu):
    A = gpu
    ref = []
    for t, e in engines(A):
        e.init_factors(0)
        ref.append(e.als(4, 0.0, graph=True)["trace"])
    pairs = engines(A)
    es = [e for _, e in pairs]
    for e in es:
        e.init_factors(0)
    b = A.BatchSweep(es)
    b.begin()
    b.time_sweeps(4)
    for e, r in zip(es, ref):
        assert abs(e.fit() - r[-1]) < 1e-5
    assert b.kernels() == sum(e.launch_counts(0)[0] for e in es)
    b.free()


def test_autotune_keeps_results(gpu):
    A = gpu
    t = A.Tensor.generate([400, 300, 200, 100], 80000, alpha=1.2, seed=7)
    plan, _, _ = A.plan_analytic(t, 16)
    e0 = A.Engine(t, 16, plan)
    e0.init_factors(0)
    r0 = e0.als(3, 0.0)
    e1 = A.Engine(t, 16, plan)
    best = e1.autotune(((32, 16), (256, 128), (1024, 512)), sweeps=2)
    assert best in (0, 1, 2)
    e1.init_factors(0)
    r1 = e1.als(3, 0.0)
    assert abs(r0["fit"] - r1["fit"]) < 1e-5
    # the same factors through both chunkings give the same MTTKRP
    import oracle as O
    mats = O.init_factors(e0.dims, 16, 3)
    e0.set_factors(mats)
    e1.set_factors(mats)
    for m in range(4):
        m0 = e0.mttkrp(m)
        m1 = e1.mttkrp(m)
        assert np.max(np.abs(m0 - m1)) <= 1e-5 * np.max(np.abs(m0))


@pytest.mark.parametrize("R", [8, 32, 64])
def test_resident_and_per_warp_grids_agree(gpu, R):
    """The contraction grid shapes (resident blocks claiming chunks from a
    counter, and one chunk per warp as batches use) give the same MTTKRP
    sequence up to FP32 summation order, on memo-root, folded and plain
    walks."""
    import oracle as O
    A = gpu
    for k, (dims, nnz, alpha) in enumerate(SHAPES):
        t = A.Tensor.generate(dims, nnz, alpha=alpha, seed=300 + k)
        plan, _, _ = A.plan_analytic(t, R)
        mats = O.init_factors(list(t.info()[2]), R, 7)
        e0 = A.Engine(t, R, plan)
        e1 = A.Engine(t, R, plan)
        e1.set_resident_grid(False)
        e0.set_factors(mats)
        e1.set_factors(mats)
        for m in range(len(dims)):
            a, b = e0.mttkrp(m), e1.mttkrp(m)
            assert np.max(np.abs(a - b)) <= 2e-5 * max(1e-30, np.max(np.abs(a))), (k, m)
        e0.free()
        e1.free()


@pytest.mark.slow
def test_batch_of_64_repeats_and_tracks_fp64():
    """The 64-tensor batch (orders 3-5, dims 100..50000, 1e4..2e6 draws,
    uniform or Zipf indices, R = 16): two batched runs of 20 iterations from
    the same start agree bit for bit, and every tensor's fit is within 1e-4
    of the FP64 run of the reference's ALS steps."""
    import subprocess
    import sys
    import json
    import os
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-m", "adatm_b200.batch_case", "--tensors", "64",
                          "--sweeps", "18", "--no-tune", "--fp64-check"], cwd=root,
                         capture_output=True, text=True, timeout=1800)
    assert out.returncode == 0, out.stderr[-2000:]
    res = json.loads(out.stdout.strip().splitlines()[-1])
    assert res["batched_reruns_identical"]
    assert res["max_fit_difference_sequential_rerun"] == 0.0
    assert res["fp64_fit_distance"]["max"] < 1e-4, res["fp64_fit_distance"]
