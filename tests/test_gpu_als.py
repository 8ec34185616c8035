"""CP-ALS on the GPU against the FP64 oracle: fit within 1e-4."""
import numpy as np
import pytest

import oracle as O
from conftest import golden_cases, load_golden
from _gen import draw_coo

pytestmark = pytest.mark.gpu

FIT_TOL = 1e-4


@pytest.mark.parametrize("name", golden_cases())
@pytest.mark.parametrize("graph", [False, True])
def test_als_fit_matches_reference(gpu, name, graph):
    A = gpu
    d = load_golden(name)
    R = int(d["R"])
    t = A.Tensor.from_coo(d["inds"], d["vals"], d["dims_list"])
    e = A.Engine(t, R, {"nmodes": d["N"], "groups": d["groups"]})
    e.init_factors(0)
    res = e.als(5, 0.0, graph=graph)
    assert res["iters"] == 5
    assert abs(res["fit"] - float(d["als5_fit"])) < FIT_TOL


@pytest.mark.parametrize("bf16", [False, True])
def test_als_trace_memo_and_plain(gpu, bf16):
    A = gpu
    inds, vals, dims = draw_coo([200, 150, 100, 50], 40000, 21, 1.1)
    ci, cv, cd = O.coo_clean(inds, vals, dims)
    cd = [int(x) for x in cd]
    R = 16
    groups, _ = O.plan(ci, cd, R)
    om = O.Model(ci, cv, cd, R, groups)
    ref = om.cpd_als(O.init_factors(cd, R, 0), 20, 0.0)
    t = A.Tensor.from_coo(ci, cv, cd)
    for plan in ({"nmodes": 4, "groups": groups}, A.plan_splatt(t, A.CSF_ALLMODE)):
        e = A.Engine(t, R, plan, bf16=bf16)
        e.init_factors(0)
        res = e.als(20, 0.0, graph=True)
        # BF16 factor rows carry 8 mantissa bits: the fit trace stays within
        # 1e-2 of FP64 (FP32 rows: 1e-4)
        tol = FIT_TOL if not bf16 else 1e-2
        assert np.max(np.abs(res["trace"] - ref["trace"])) < tol
        mats, lam = e.get_factors()
        assert np.all(np.isfinite(lam))


def test_als_tolerance_stops_early(gpu):
    A = gpu
    inds, vals, dims = draw_coo([30, 30, 30], 3000, 2)
    ci, cv, cd = O.coo_clean(inds, vals, dims)
    cd = [int(x) for x in cd]
    groups, _ = O.plan(ci, cd, 4)
    om = O.Model(ci, cv, cd, 4, groups)
    ref = om.cpd_als(O.init_factors(cd, 4, 0), 200, 1e-3)
    t = A.Tensor.from_coo(ci, cv, cd)
    e = A.Engine(t, 4, {"nmodes": 3, "groups": groups})
    e.init_factors(0)
    res = e.als(200, 1e-3, graph=True)
    assert abs(res["iters"] - ref["iters"]) <= 1
    assert res["iters"] < 200


def test_planted_low_rank(gpu):
    A = gpu
    rng = np.random.default_rng(8)
    dims = [20, 18, 16]
    R = 3
    fac = [rng.random((d, R)) for d in dims]
    grid = np.array(np.meshgrid(*[np.arange(d) for d in dims], indexing="ij")).reshape(3, -1)
    vals = np.einsum("ir,ir,ir->i", fac[0][grid[0]], fac[1][grid[1]], fac[2][grid[2]])
    vals = vals * (1 + 0.001 * rng.standard_normal(vals.size))
    t = A.Tensor.from_coo(grid.astype(np.uint64), vals, dims)
    plan, _, _ = A.plan_analytic(t, R)
    e = A.Engine(t, R, plan)
    e.init_factors(1)
    res = e.als(200, 0.0, graph=True)
    assert res["fit"] > 0.99


@pytest.mark.parametrize("rows,R", [(1, 1), (1000, 16), (5000, 32), (20000, 64), (777, 100)])
def test_gram_device_entry_point(gpu, rows, R):
    import torch
    A = gpu
    ldr = (R + 3) // 4 * 4
    x = torch.rand(rows, ldr, device="cuda", dtype=torch.float32, generator=torch.Generator("cuda").manual_seed(rows))
    x[:, R:] = 0
    G = torch.zeros(R, R, device="cuda", dtype=torch.float64)
    A.gram_device(x.data_ptr(), rows, R, ldr, G.data_ptr())
    ref = x[:, :R].double().T @ x[:, :R].double()
    # TF32 tensor-core tiles (three-term split) with FP32 sums per 8 rows
    assert torch.allclose(G, ref, rtol=1e-6, atol=1e-6 * float(ref.abs().max()))


def test_bf16_sweep_fit_tracks_fp32(gpu):
    """BF16 gathers with the fit's MTTKRP in FP32: fit stays finite and close
    to the FP32 sweep on a skewed 4-mode tensor."""
    A = gpu
    t = A.Tensor.generate([5000, 5000, 2000, 500], 3_000_000, alpha=1.1, seed=0)
    plan, _, _ = A.plan_analytic(t, 32)
    res = {}
    for bf in (False, True):
        e = A.Engine(t, 32, plan, bf16=bf)
        e.init_factors(0)
        res[bf] = e.als(8, 0.0, graph=True)["trace"]
    assert np.all(np.isfinite(res[True]))
    assert np.max(np.abs(res[True] - res[False])) < 1e-2
