"""The sharded sweep's GPU data path (adatm_b200.shard with engines): three
shards of one tensor on one device, summed locally, give the single-engine
sweep and stay within the fit bar of the FP64 oracle."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bf16", [False, True])
def test_virtual_shards_match_one_engine(gpu, bf16):
    import torch
    from adatm_b200 import shard as S
    A = gpu
    R = 16
    full = A.Tensor.generate([800, 600, 300, 120], 400000, alpha=1.2, seed=5)
    inds, vals, dims = full.download()
    plan = A.plan_analytic(full, R)[0]
    one = A.Engine(full, R, plan, bf16=bf16)
    one.init_factors(0)
    ref = one.als(6, 0.0, graph=False)["trace"]
    shards, tensors = [], []
    for r in range(3):
        li, lv = S.shard_coo(inds, vals, 3, r)
        t = A.Tensor.from_coo(li, lv, dims)
        e = A.Engine(t, R, plan, bf16=bf16)
        e.init_factors(0)
        tensors.append(t)
        shards.append(e)
    ldr = (R + 3) // 4 * 4
    bufs = S.torch_buffers(dims, 3, ldr, "cuda")
    cpd = S.ShardedCpd(shards, len(dims), bufs, lambda b: b.data_ptr(), S.local_allreduce)
    trace = np.array(cpd.als(6))
    assert np.max(np.abs(trace - ref)) < 2e-5, (trace, ref)
    if not bf16:
        start = [np.asarray(m, dtype=np.float32).astype(np.float64) for m in O.init_factors(dims, R, 0)]
        fp64 = O.cpd_als_coo(inds, vals, dims, R, start, 6, 0.0)["trace"]
        assert np.max(np.abs(trace - fp64)) < 1e-4
