"""Deterministic accumulation (adatm_engine_set_deterministic): no float
atomics in any MTTKRP. The results equal the FP64 oracle within the FP32
bound, and repeated runs -- MTTKRP sequences, ALS fit traces, batched
sweeps -- agree bit for bit."""
import numpy as np
import pytest

import oracle as O
from conftest import golden_cases, load_golden
from _gen import draw_coo

pytestmark = pytest.mark.gpu

TOL_F32 = 2e-5


def rel_err(a, b):
    return float(np.max(np.abs(a - b)) / max(1e-30, np.max(np.abs(b))))


@pytest.mark.parametrize("name", golden_cases())
def test_golden_sequence(gpu, name):
    A = gpu
    d = load_golden(name)
    N, R = d["N"], int(d["R"])
    t = A.Tensor.from_coo(d["inds"], d["vals"], d["dims_list"])
    e = A.Engine(t, R, {"nmodes": N, "groups": d["groups"]})
    e.set_deterministic(True)
    mats = O.init_factors(d["dims_list"], R, 0)
    e.set_factors(mats)
    for it in range(2):
        for m in range(N):
            assert rel_err(e.mttkrp(m), d[f"mttkrp_it{it}_m{m}"]) < TOL_F32, (it, m)


@pytest.mark.parametrize("R", [5, 16, 32, 64, 100])
@pytest.mark.parametrize("chunk", [0, 3, 40])
def test_every_plan_kind(gpu, R, chunk):
    """Memo roots, memo reuse (scatters and contractions below the root),
    recomputes from the leaves, with chunks cutting nodes at every level and
    skewed rows long enough to be split into pieces."""
    A = gpu
    inds, vals, dims = draw_coo([60, 40, 30, 25, 12], 60000, 21, 1.6)
    ci, cv, cd = O.coo_clean(inds, vals, dims)
    cd = [int(x) for x in cd]
    t = A.Tensor.from_coo(ci, cv, cd)
    _, cands, _ = A.plan_analytic(t, R)
    mats = O.init_factors(cd, R, 2)
    for c in cands:
        e = A.Engine(t, R, c, chunk_leaf=chunk, chunk_rows=chunk)
        e.set_deterministic(True)
        e.set_factors(mats)
        om = O.Model(ci, cv, cd, R, c["groups"])
        for m in range(5):
            want = om.mttkrp(mats, m)
            assert rel_err(e.mttkrp(m), want) < TOL_F32, (c["groups"], m)
            assert rel_err(e.mttkrp_direct(m), want) < TOL_F32, (c["groups"], m)
        e.free()


@pytest.mark.parametrize("walkers", [1, 2, 4])
def test_repeats_bit_for_bit(gpu, walkers):
    A = gpu
    t = A.Tensor.generate([3000, 2000, 800, 300], 2_000_000, alpha=1.3, seed=9)
    plan, _, _ = A.plan_analytic(t, 32)
    e = A.Engine(t, 32, plan)
    e.set_walkers(walkers)
    e.set_deterministic(True)
    mats = O.init_factors(e.dims, 32, 4)
    runs = []
    for _ in range(3):
        e.set_factors(mats)
        runs.append([e.mttkrp(m).tobytes() for m in range(4)])
    assert runs[0] == runs[1] == runs[2]
    traces = []
    for _ in range(2):
        e.init_factors(0)
        traces.append(e.als(8, 0.0, graph=True)["trace"].tobytes())
    assert traces[0] == traces[1]
    # same numbers as the atomic mode, up to FP32 summation order
    e.init_factors(0)
    det = e.als(3, 0.0, graph=False)["fit"]
    e.set_deterministic(False)
    e.init_factors(0)
    atom = e.als(3, 0.0, graph=False)["fit"]
    assert abs(det - atom) < 1e-5


def test_batched_sweeps_repeat(gpu):
    A = gpu
    shapes = [([300, 200, 100], 20000, None), ([120, 90, 80, 70], 30000, 1.2),
              ([60, 50, 40, 30, 20], 25000, 1.1), ([2000, 1500, 900], 60000, 1.3)]
    es, ts = [], []
    for k, (dims, nnz, alpha) in enumerate(shapes):
        t = A.Tensor.generate(dims, nnz, alpha=alpha, seed=300 + k)
        plan, _, _ = A.plan_analytic(t, 16)
        e = A.Engine(t, 16, plan)
        e.set_deterministic(True)
        ts.append(t)
        es.append(e)
    fits = []
    for _ in range(2):
        for e in es:
            e.init_factors(0)
        b = A.BatchSweep(es)
        b.begin()
        b.time_sweeps(6)
        fits.append([e.fit() for e in es])
        b.free()
    assert fits[0] == fits[1]
