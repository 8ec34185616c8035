"""Parity at the full sizes of the benchmark configurations (the seeded
synthetic stand-ins for them): the device generator equals its host port, the
trees the plan builds are bit-exact with the oracle's, every mode's MTTKRP is
within the FP32 / BF16 bounds of the FP64 oracle, and the fit after the
configuration's full sweep count is within 1e-4 of the FP64 run from the
same start (the reference's ALS steps, cpd_als_iterate_adaptive,
adatm_cpd.c:256-373, with the FP64 COO MTTKRP)."""
import numpy as np
import pytest

import oracle as O

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

CONFIGS = {
    # 1000^3, 1M uniform draws, R = 16, 10 sweeps
    "uniform_3mode": dict(dims=[1000, 1000, 1000], nnz=1_000_000, alpha=None, vk=0, R=16, iters=10),
    # 5000 x 5000 x 2000 x 500, 20M Zipf(1.1) draws, R = 32, 20 sweeps
    "zipf_4mode": dict(dims=[5000, 5000, 2000, 500], nnz=20_000_000, alpha=1.1, vk=0, R=32, iters=20),
    # 20000 x 10000 x 5000 x 1000 x 200, 50M Zipf(1.2) draws, lognormal values, R = 64
    "bf16_5mode": dict(dims=[20000, 10000, 5000, 1000, 200], nnz=50_000_000, alpha=1.2, vk=1, R=64,
                       iters=20),
}
FIT_TOL = 1e-4        # |fit_gpu - fit_fp64| after the configuration's sweeps
MTTKRP_F32 = 2e-5     # ||M_gpu - M_fp64|| / ||M_fp64||, FP32 rows
MTTKRP_ACC = 2e-5     # BF16 rows vs FP64 on the same (BF16-valued) factors: FP32 accumulation
MTTKRP_BF16 = 4e-3    # BF16-rounded start factors vs the unrounded FP64 run (quantisation)

_cache = {}


def workload(A, name):
    if name not in _cache:  # every workload is built once per session
        c = CONFIGS[name]
        O.threads(0)
        t = A.Tensor.generate(c["dims"], c["nnz"], alpha=c["alpha"], value_kind=c["vk"], seed=0)
        inds, vals, dims = t.download()
        plan = A.plan_analytic(t, c["R"])[0]
        _cache[name] = (t, inds, vals, dims, plan)
    return _cache[name]


def start32(dims, R):
    return [np.asarray(m, dtype=np.float32).astype(np.float64) for m in O.init_factors(dims, R, 0)]


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("name", list(CONFIGS))
def test_generator_equals_host_port(gpu, name):
    t, inds, vals, dims, _ = workload(gpu, name)
    c = CONFIGS[name]
    hi, hv, hd = O.generate(c["dims"], c["nnz"], alpha=c["alpha"], value_kind=c["vk"], seed=0)
    assert hd == dims
    assert hi.tobytes() == inds.tobytes()
    if c["vk"] == 0:
        assert hv.tobytes() == vals.tobytes()
    else:  # lognormal: the device's exp / log / cos round differently
        assert np.max(np.abs(hv - vals) / np.abs(hv)) < 1e-12


@pytest.mark.parametrize("name", ["uniform_3mode", "zipf_4mode"])
def test_trees_bit_exact_full_size(gpu, name):
    A = gpu
    t, inds, vals, dims, plan = workload(A, name)
    e = A.Engine(t, CONFIGS[name]["R"], plan)
    N = len(dims)
    for g, gr in enumerate(plan["groups"]):
        got = e.csf_arrays(g)
        ref = O.csf_build(inds, vals, dims, gr["o_opt"])
        np.testing.assert_array_equal(got["nfibs"], ref["nfibs"])
        for l in range(N - 1):
            np.testing.assert_array_equal(got["fptr"][l], ref["fptr"][l])
        for l in range(1, N):
            np.testing.assert_array_equal(got["fids"][l], ref["fids"][l])
        assert got["vals"].tobytes() == ref["vals"].tobytes()
    e.free()


@pytest.mark.parametrize("name", list(CONFIGS))
@pytest.mark.parametrize("bf16", [False, True])
def test_mttkrp_each_mode_full_size(gpu, name, bf16):
    """Every mode's MTTKRP of the plan's sequence (memo roots store their
    rows, reuse modes read them) against the FP64 COO MTTKRP."""
    A = gpu
    t, inds, vals, dims, plan = workload(A, name)
    R = CONFIGS[name]["R"]
    e = A.Engine(t, R, plan, bf16=bf16)
    start = start32(dims, R)
    e.set_factors(start)
    used = e.get_factors()[0]  # the factor values the device holds (BF16-valued with bf16)
    for m in range(len(dims)):
        got = e.mttkrp(m)
        if bf16:
            assert rel(got, O.mttkrp_coo(inds, vals, dims, used, m, R)) < MTTKRP_ACC, m
            assert rel(got, O.mttkrp_coo(inds, vals, dims, start, m, R)) < MTTKRP_BF16, m
        else:
            assert rel(got, O.mttkrp_coo(inds, vals, dims, start, m, R)) < MTTKRP_F32, m
    e.free()


@pytest.mark.parametrize("name,bf16", [(n, False) for n in CONFIGS] + [("bf16_5mode", True)])
def test_fit_after_full_sweeps(gpu, name, bf16):
    A = gpu
    t, inds, vals, dims, plan = workload(A, name)
    c = CONFIGS[name]
    e = A.Engine(t, c["R"], plan, bf16=bf16)
    e.init_factors(0)
    got = e.als(c["iters"], 0.0, graph=True)
    e.free()
    ref = O.cpd_als_coo(inds, vals, dims, c["R"], start32(dims, c["R"]), c["iters"], 0.0)
    assert got["iters"] == c["iters"]
    assert abs(got["fit"] - ref["fit"]) < FIT_TOL, (got["trace"] - ref["trace"]).tolist()
