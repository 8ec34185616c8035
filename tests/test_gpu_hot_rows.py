"""Atomic scatter walks (deterministic accumulation off) whose output rows
are hit by very many units sum those rows per block in shared memory; the
MTTKRP must not change (FP32 summation order aside). Tensors are built so that one output row takes about half of the
units of a leaf scatter and of a memo-reuse scatter (the hot mode has a
large dimension, so plans place it below the root, where it is scattered).
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

TOL_F32 = 2e-5


def skewed(dims, nnz, hot_mode, seed):
    rng = np.random.default_rng(seed)
    inds = np.stack([rng.integers(0, d, nnz) for d in dims]).astype(np.uint64)
    inds[hot_mode, rng.random(nnz) < 0.5] = 3  # row 3 of the hot mode
    vals = rng.random(nnz)
    ci, cv, cd = O.coo_clean(inds, vals, dims)
    return ci, cv, [int(x) for x in cd]


def rel_err(a, b):
    return float(np.max(np.abs(a - b)) / max(1e-30, np.max(np.abs(b))))


@pytest.mark.parametrize("R", [16, 32])
@pytest.mark.parametrize("case", [([60000, 40, 30], 400000, 1), ([400, 300, 50000], 300000, 2),
                                  ([300, 250, 60000, 20], 400000, 2)])
def test_hot_output_rows(gpu, R, case):
    A = gpu
    dims, nnz, hot = case
    ci, cv, cd = skewed(dims, nnz, hot, 11)
    t = A.Tensor.from_coo(ci, cv, cd)
    mats = O.init_factors(cd, R, 5)
    plans = [A.plan_splatt(t, alloc) for alloc in (0, 1, 2)]
    _, cands, _ = A.plan_analytic(t, R)
    plans += [{"nmodes": c["nmodes"], "groups": c["groups"]} for c in cands]
    hot_walks = 0
    for plan in plans:
        e = A.Engine(t, R, plan)
        e.set_deterministic(False)
        e.set_factors(mats)
        om = O.Model(ci, cv, cd, R, plan["groups"]) if "use_csfs" not in plan else None
        for m in range(len(cd)):
            hot_walks += e.hot_rows(m) > 0
            if om is not None:
                ref = om.mttkrp(mats, m)
            else:
                g = plan["use_csfs"][m]
                ref = O.mttkrp_csf(ci, cv, cd, plan["groups"][g]["o_opt"], mats, m, R)
            assert rel_err(e.mttkrp(m), ref) < TOL_F32, (plan, m)
            assert rel_err(e.mttkrp_direct(m), ref) < TOL_F32, (plan, m)
        e.free()
    assert hot_walks > 0
