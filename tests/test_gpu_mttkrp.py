"""MTTKRP kernels (memo root, memo reuse, recompute, plain root) against the
FP64 oracle; FP32 accumulation, FP32 or BF16 factor gathers."""
import numpy as np
import pytest

import oracle as O
from conftest import golden_cases, load_golden
from _gen import draw_coo

pytestmark = pytest.mark.gpu

TOL_F32 = 2e-5   # max |gpu - oracle| / max |oracle|, FP32 gathers
TOL_BF16 = 3e-2  # BF16 factor rows (8-bit mantissa) with FP32 accumulation


def rel_err(a, b):
    return float(np.max(np.abs(a - b)) / max(1e-30, np.max(np.abs(b))))


@pytest.mark.parametrize("name", golden_cases())
@pytest.mark.parametrize("bf16", [False, True])
def test_memo_sequence_matches_reference(gpu, name, bf16):
    A = gpu
    d = load_golden(name)
    N, R = d["N"], int(d["R"])
    t = A.Tensor.from_coo(d["inds"], d["vals"], d["dims_list"])
    e = A.Engine(t, R, {"nmodes": N, "groups": d["groups"]}, bf16=bf16)
    mats = O.init_factors(d["dims_list"], R, 0)
    e.set_factors(mats)
    tol = TOL_BF16 if bf16 else TOL_F32
    for it in range(2):
        for m in range(N):
            assert rel_err(e.mttkrp(m), d[f"mttkrp_it{it}_m{m}"]) < tol, (it, m)


@pytest.mark.parametrize("name", golden_cases())
def test_memo_rows_match_oracle(gpu, name):
    A = gpu
    d = load_golden(name)
    N, R = d["N"], int(d["R"])
    t = A.Tensor.from_coo(d["inds"], d["vals"], d["dims_list"])
    e = A.Engine(t, R, {"nmodes": N, "groups": d["groups"]})
    mats = O.init_factors(d["dims_list"], R, 1)
    e.set_factors(mats)
    om = O.Model(d["inds"], d["vals"], d["dims_list"], R, d["groups"])
    for g, gr in enumerate(d["groups"]):
        if gr["n_imten"] == 0:
            continue
        e.mttkrp(gr["memo_mode"])
        om.mttkrp(mats, gr["memo_mode"])
        # the oracle keeps memo rows internally; rebuild them from its tree
        ct = O.csf_build(d["inds"], d["vals"], d["dims_list"], gr["o_opt"])
        for deg in range(gr["n_imten"]):
            lvl = gr["begin_imten"] - 1 - deg
            rows = e.memo(g, deg)
            ref = _level_sums(ct, mats, lvl, R)
            assert rel_err(rows, ref) < TOL_F32, (g, deg)


def _level_sums(ct, mats, lvl, R):
    N = ct["nmodes"]
    perm = [int(x) for x in ct["dim_perm"]]
    F = [int(x) for x in ct["nfibs"]]
    cur = np.zeros((F[N - 2], R))
    U = mats[perm[N - 1]]
    fp = ct["fptr"][N - 2]
    for f in range(F[N - 2]):
        s, e = int(fp[f]), int(fp[f + 1])
        cur[f] = (ct["vals"][s:e, None] * U[ct["fids"][N - 1][s:e].astype(np.int64)]).sum(0)
    lev = N - 2
    while lev > lvl:
        nxt = np.zeros((F[lev - 1], R))
        U = mats[perm[lev]]
        fp = ct["fptr"][lev - 1]
        for s in range(F[lev - 1]):
            a, b = int(fp[s]), int(fp[s + 1])
            nxt[s] = (cur[a:b] * U[ct["fids"][lev][a:b].astype(np.int64)]).sum(0)
        cur = nxt
        lev -= 1
    return cur


@pytest.mark.parametrize("alloc", [0, 1, 2])
@pytest.mark.parametrize("dims,alpha,R", [([60, 50, 40], None, 16), ([40, 30, 20, 25], 1.2, 32),
                                          ([12, 10, 9, 11, 8], 1.1, 10), ([8, 7, 6, 9, 5, 6], None, 64)])
def test_plain_splatt_allocations(gpu, alloc, dims, alpha, R):
    """ONEMODE/TWOMODE/ALLMODE plans: root, internal and leaf kernels."""
    A = gpu
    inds, vals, dims = draw_coo(dims, 6000, 42, alpha)
    ci, cv, cd = O.coo_clean(inds, vals, dims)
    cd = [int(x) for x in cd]
    t = A.Tensor.from_coo(ci, cv, cd)
    plan = A.plan_splatt(t, alloc)
    e = A.Engine(t, R, plan)
    mats = O.init_factors(cd, R, 2)
    e.set_factors(mats)
    for m in range(len(cd)):
        g = plan["use_csfs"][m]
        ref = O.mttkrp_csf(ci, cv, cd, plan["groups"][g]["o_opt"], mats, m, R)
        assert rel_err(e.mttkrp(m), ref) < TOL_F32, m


@pytest.mark.parametrize("chunk", [1, 3, 7, 32, 100, 1000])
def test_chunk_boundaries(gpu, chunk):
    """Chunks cut nodes at every level; results must not depend on the cut."""
    A = gpu
    inds, vals, dims = draw_coo([30, 20, 15, 10, 8], 20000, 9, 1.5)
    ci, cv, cd = O.coo_clean(inds, vals, dims)
    cd = [int(x) for x in cd]
    R = 8
    groups, _ = O.plan(ci, cd, R)
    t = A.Tensor.from_coo(ci, cv, cd)
    e = A.Engine(t, R, {"nmodes": 5, "groups": groups}, chunk_leaf=chunk, chunk_rows=chunk)
    om = O.Model(ci, cv, cd, R, groups)
    mats = O.init_factors(cd, R, 4)
    e.set_factors(mats)
    for m in range(5):
        assert rel_err(e.mttkrp(m), om.mttkrp(mats, m)) < TOL_F32, m
        assert rel_err(e.mttkrp_direct(m), om.mttkrp(mats, m)) < TOL_F32, m


def test_every_candidate_plan(gpu):
    """Every plan the planner enumerates, including partial memo plans the
    reference mis-computes, gives the oracle's MTTKRP sequence."""
    A = gpu
    inds, vals, dims = draw_coo([12, 11, 10, 9, 8, 7], 8000, 5, 1.1)
    ci, cv, cd = O.coo_clean(inds, vals, dims)
    cd = [int(x) for x in cd]
    R = 8
    t = A.Tensor.from_coo(ci, cv, cd)
    _, cands, _ = A.plan_analytic(t, R)
    assert len(cands) == 7
    mats = O.init_factors(cd, R, 6)
    for c in cands:
        e = A.Engine(t, R, c)
        e.set_factors(mats)
        om = O.Model(ci, cv, cd, R, c["groups"])
        for m in range(6):
            assert rel_err(e.mttkrp(m), om.mttkrp(mats, m)) < TOL_F32


@pytest.mark.parametrize("R", [1, 3, 16, 17, 33, 64, 100, 128])
def test_ranks(gpu, R):
    A = gpu
    inds, vals, dims = draw_coo([50, 40, 30, 20], 5000, 11, 1.0)
    ci, cv, cd = O.coo_clean(inds, vals, dims)
    cd = [int(x) for x in cd]
    groups, _ = O.plan(ci, cd, R)
    t = A.Tensor.from_coo(ci, cv, cd)
    e = A.Engine(t, R, {"nmodes": 4, "groups": groups})
    om = O.Model(ci, cv, cd, R, groups)
    mats = O.init_factors(cd, R, 1)
    e.set_factors(mats)
    for m in range(4):
        assert rel_err(e.mttkrp(m), om.mttkrp(mats, m)) < TOL_F32


def test_analytic_plan_matches_oracle(gpu):
    A = gpu
    for name in golden_cases():
        d = load_golden(name)
        t = A.Tensor.from_coo(d["inds"], d["vals"], d["dims_list"])
        plan, cands, chosen = A.plan_analytic(t, int(d["R"]))
        assert plan["groups"] == d["groups"], name
        _, ocfg = O.plan(d["inds"], d["dims_list"], int(d["R"]))
        assert [(c["pspace"], c["pops"]) for c in cands] == [(c["pspace"], c["pops"]) for c in ocfg]


@pytest.mark.parametrize("R", [5, 16, 32, 48, 64, 100])
@pytest.mark.parametrize("walkers", [1, 2, 4])
def test_walker_split(gpu, R, walkers):
    """The contraction source loop split into 1, 2 or 4 walkers per warp
    (segments joined once per batch) gives the oracle's MTTKRP sequence on
    every plan kind, with chunks that cut nodes at every level; walker counts
    that cannot cover the rank are refused."""
    A = gpu
    inds, vals, dims = draw_coo([40, 30, 25, 20, 12], 30000, 17, 1.3)
    ci, cv, cd = O.coo_clean(inds, vals, dims)
    cd = [int(x) for x in cd]
    t = A.Tensor.from_coo(ci, cv, cd)
    _, cands, _ = A.plan_analytic(t, R)
    mats = O.init_factors(cd, R, 3)
    ok = {(1, 1): R <= 128, (1, 2): R <= 64, (1, 4): R <= 32}[(1, walkers)]
    for c in cands[:3]:
        for chunk in (0, 7):
            e = A.Engine(t, R, c, chunk_leaf=chunk, chunk_rows=chunk)
            if not ok:
                with pytest.raises(A.AdatmError):
                    e.set_walkers(walkers)
                e.free()
                return
            e.set_walkers(walkers)
            e.set_factors(mats)
            om = O.Model(ci, cv, cd, R, c["groups"])
            for m in range(5):
                want = om.mttkrp(mats, m)
                assert rel_err(e.mttkrp(m), want) < TOL_F32, (m, chunk)
                assert rel_err(e.mttkrp_direct(m), want) < TOL_F32, (m, chunk)
            e.free()


@pytest.mark.parametrize("R", [16, 32, 64])
@pytest.mark.parametrize("fold", [0, 1, 2])
@pytest.mark.parametrize("shape", [([40, 30, 25, 20, 12], 30000), ([900, 700, 500, 300, 200], 40000)])
def test_folded_levels(gpu, R, fold, shape):
    """Contractions with 0, 1 or 2 unstored levels folded into the source
    loop (each unit multiplied by its ancestors' rows) give the oracle's
    MTTKRP sequence on the plain all-mode plan (leaf-to-root walks with no
    stores, where two levels fold), the one-mode plan (folded walks that end
    below the root) and on memo plans, with chunks that cut
    nodes at every level, deterministic and atomic, at every walker count
    that covers the rank."""
    A = gpu
    dims, nnz = shape
    inds, vals, dims = draw_coo(dims, nnz, 23, 1.2)
    ci, cv, cd = O.coo_clean(inds, vals, dims)
    cd = [int(x) for x in cd]
    t = A.Tensor.from_coo(ci, cv, cd)
    _, cands, _ = A.plan_analytic(t, R)
    plans = [A.plan_splatt(t, A.CSF_ALLMODE), A.plan_splatt(t, A.CSF_ONEMODE)]
    plans += [{"nmodes": c["nmodes"], "groups": c["groups"]} for c in cands[:2]]
    mats = O.init_factors(cd, R, 4)
    walkers = [w for w in (1, 2, 4) if (32 // w) * 4 >= R]
    for p, plan in enumerate(plans):
        om = O.Model(ci, cv, cd, R, plan["groups"]) if "use_csfs" not in plan else None
        for chunk in (0, 7):
            for det in (True, False):
                e = A.Engine(t, R, plan, chunk_leaf=chunk, chunk_rows=chunk)
                e.set_fold(fold)
                e.set_deterministic(det)
                e.set_walkers(walkers[(p + chunk) % len(walkers)])
                e.set_factors(mats)
                for m in range(5):
                    if om is not None:
                        want = om.mttkrp(mats, m)
                    else:
                        g = plan["use_csfs"][m]
                        want = O.mttkrp_csf(ci, cv, cd, plan["groups"][g]["o_opt"], mats, m, R)
                    assert rel_err(e.mttkrp(m), want) < TOL_F32, (p, m, chunk, det)
                e.free()


def test_fold_refused(gpu):
    """Fold counts outside -1..2 are refused."""
    A = gpu
    inds, vals, dims = draw_coo([40, 30, 25], 3000, 5, 1.2)
    ci, cv, cd = O.coo_clean(inds, vals, dims)
    t = A.Tensor.from_coo(ci, cv, [int(x) for x in cd])
    e = A.Engine(t, 16, A.plan_splatt(t, A.CSF_ALLMODE))
    for bad in (-2, 3):
        with pytest.raises(A.AdatmError):
            e.set_fold(bad)
    e.free()
