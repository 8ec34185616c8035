"""The oracle restatement against the reference's own outputs (golden
fixtures made by running the reference's C files) and against brute force."""
import numpy as np
import pytest

import oracle as O
from conftest import golden_cases, load_golden
from _gen import draw_coo, dense_mttkrp


@pytest.mark.parametrize("name", golden_cases())
def test_plan_matches_reference(name):
    d = load_golden(name)
    groups, configs = O.plan(d["inds"], d["dims_list"], int(d["R"]))
    assert groups == d["groups"]
    uc, ut = O.decide_use_csfs(d["N"], groups)
    np.testing.assert_array_equal(uc, d["use_csfs"])
    np.testing.assert_array_equal(ut, d["use_tags"])


@pytest.mark.parametrize("name", golden_cases())
def test_csf_bit_exact_with_reference(name):
    d = load_golden(name)
    N = d["N"]
    for g, gr in enumerate(d["groups"]):
        c = O.csf_build(d["inds"], d["vals"], d["dims_list"], gr["o_opt"])
        np.testing.assert_array_equal(c["nfibs"], d[f"g{g}_nfibs"])
        assert c["vals"].tobytes() == d[f"g{g}_vals"].tobytes()
        for l in range(N - 1):
            np.testing.assert_array_equal(c["fptr"][l], d[f"g{g}_fptr{l}"])
        for l in range(1, N):
            np.testing.assert_array_equal(c["fids"][l], d[f"g{g}_fids{l}"])
        assert f"g{g}_fids0" not in d  # the reference keeps fids[0] NULL


@pytest.mark.parametrize("name", golden_cases())
def test_mttkrp_sequence_matches_reference(name):
    d = load_golden(name)
    N, R = d["N"], int(d["R"])
    md = O.Model(d["inds"], d["vals"], d["dims_list"], R, d["groups"])
    mats = O.init_factors(d["dims_list"], R, 0)
    for it in range(2):
        for m in range(N):
            got = md.mttkrp(mats, m)
            ref = d[f"mttkrp_it{it}_m{m}"]
            assert np.max(np.abs(got - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref)))


@pytest.mark.parametrize("name", golden_cases())
def test_cpd_als_matches_reference(name):
    d = load_golden(name)
    R = int(d["R"])
    md = O.Model(d["inds"], d["vals"], d["dims_list"], R, d["groups"])
    res = md.cpd_als(O.init_factors(d["dims_list"], R, 0), 5, 0.0)
    assert abs(res["fit"] - float(d["als5_fit"])) < 1e-12
    np.testing.assert_allclose(res["lambda"], d["als5_lambda"], rtol=1e-10)


@pytest.mark.parametrize("N,dims", [(3, [9, 8, 7]), (4, [7, 6, 5, 8]), (5, [5, 4, 6, 5, 4]),
                                    (6, [4, 3, 4, 5, 3, 4])])
def test_oracle_against_brute_force(N, dims):
    inds, vals, dims = draw_coo(dims, 400, seed=N)
    inds, vals, dims = O.coo_clean(inds, vals, dims)
    dims = [int(x) for x in dims]
    R = 5
    groups, _ = O.plan(inds, dims, R)
    md = O.Model(inds, vals, dims, R, groups)
    mats = O.init_factors(dims, R, 3)
    for m in range(N):
        ref = dense_mttkrp(inds, vals, dims, mats, m)
        np.testing.assert_allclose(md.mttkrp(mats, m), ref, rtol=1e-12, atol=1e-12)
        perm = O.splatt_perm(dims, 1, m)
        np.testing.assert_allclose(O.mttkrp_csf(inds, vals, dims, perm, mats, m, R), ref,
                                   rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("N,expected", [(3, 1), (4, 3), (5, 4), (6, 7), (7, 8), (8, 11)])
def test_candidate_counts(N, expected):
    assert len(O.candidate_configs([10 + m for m in range(N)])) == expected


def test_pair_sort_sorts_and_keeps_reference_tie_order():
    rng = np.random.default_rng(0)
    for n in range(1, 12):
        for _ in range(50):
            y = rng.integers(0, 4, n)
            x = np.arange(n)
            xs, ys = O.pair_sort(x, y)
            assert np.all(np.diff(ys.astype(np.int64)) >= 0)
            assert sorted(xs.tolist()) == list(range(n))
    # three equal keys rotate as the reference's quicksort does
    xs, _ = O.pair_sort([7, 8, 9], [5, 5, 5])
    assert xs.tolist() == [9, 7, 8]


def test_coo_clean_sums_duplicates_in_order_and_compacts():
    inds = np.array([[3, 1, 3, 3], [0, 2, 0, 5], [4, 4, 4, 4]], dtype=np.uint64)
    vals = np.array([0.1, 0.2, 0.3, 0.4])
    ci, cv, cd = O.coo_clean(inds, vals, [5, 6, 7])
    assert list(cd) == [2, 3, 1]
    assert ci.shape == (3, 3)
    np.testing.assert_array_equal(ci[0], [0, 1, 1])
    np.testing.assert_array_equal(ci[1], [1, 0, 2])
    assert cv[1] == 0.1 + 0.3


def test_planted_rank_one_fit_goes_to_one():
    rng = np.random.default_rng(3)
    dims = [12, 10, 9, 8]
    a = [rng.random(d) + 0.1 for d in dims]
    grid = np.array(np.meshgrid(*[np.arange(d) for d in dims], indexing="ij")).reshape(4, -1)
    vals = a[0][grid[0]] * a[1][grid[1]] * a[2][grid[2]] * a[3][grid[3]]
    vals = vals * (1 + 0.01 * rng.standard_normal(vals.size))
    inds = grid.astype(np.uint64)
    groups, _ = O.plan(inds, dims, 1)
    md = O.Model(inds, vals, dims, 1, groups)
    res = md.cpd_als(O.init_factors(dims, 1, 0), 20, 0.0)
    # an exact rank-1 tensor drives the residual to rounding noise, where the
    # reference's sqrt(||X||^2 + ||Z||^2 - 2<X,Z>) may turn NaN; 1% noise
    # keeps the fit just below 1
    assert 0.985 < res["fit"] < 1.0


def test_empty_and_single_nonzero_csf():
    c = O.csf_build(np.zeros((3, 0), dtype=np.uint64), np.zeros(0), [2, 2, 2], [0, 1, 2])
    assert list(c["nfibs"]) == [0, 0, 0]
    c = O.csf_build(np.array([[1], [0], [2]], dtype=np.uint64), np.array([2.5]), [2, 1, 3], [2, 0, 1])
    assert list(c["nfibs"]) == [1, 1, 1]
    assert list(c["fptr"][0]) == [0, 1] and list(c["fptr"][1]) == [0, 1]
    assert list(c["fids"][2]) == [0] and c["vals"][0] == 2.5


@pytest.mark.parametrize("name", golden_cases())
def test_coo_path_matches_tree_restatement(name):
    """The OpenMP COO MTTKRP and the ALS built on it (the FP64 reference run
    for full-size workloads) equal the tree restatement, which the golden
    fixtures pin to the reference's own code."""
    d = load_golden(name)
    N, R = d["N"], int(d["R"])
    md = O.Model(d["inds"], d["vals"], d["dims_list"], R, d["groups"])
    mats = O.init_factors(d["dims_list"], R, 0)
    for m in range(N):
        a = md.mttkrp(mats, m)
        b = O.mttkrp_coo(d["inds"], d["vals"], d["dims_list"], mats, m, R)
        assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(a))
    r1 = md.cpd_als(mats, 5, 0.0)
    r2 = O.cpd_als_coo(d["inds"], d["vals"], d["dims_list"], R, mats, 5, 0.0)
    assert abs(r1["fit"] - r2["fit"]) < 1e-12
    assert abs(r2["fit"] - float(d["als5_fit"])) < 1e-10
    np.testing.assert_allclose(r2["lambda"], r1["lambda"], rtol=1e-9)


def test_coo_path_repeats_at_fixed_threads():
    inds, vals, dims = O.generate([300, 200, 100, 50], 200_000, alpha=1.2, seed=5)
    mats = O.init_factors(dims, 8, 1)
    a = O.mttkrp_coo(inds, vals, dims, mats, 2, 8)
    b = O.mttkrp_coo(inds, vals, dims, mats, 2, 8)
    assert a.tobytes() == b.tobytes()


@pytest.mark.parametrize("alpha,kind", [(None, 0), (1.1, 0), (1.3, 1)])
def test_host_generator(alpha, kind):
    """The host port of the seeded generator: shapes, bounds, cleaned (no
    duplicates, no empty slices), deterministic; Zipf skews towards index 0;
    lognormal values are positive with log-mean near 0."""
    dims = [400, 300, 200, 100]
    inds, vals, d = O.generate(dims, 300_000, alpha=alpha, value_kind=kind, seed=11)
    i2, v2, d2 = O.generate(dims, 300_000, alpha=alpha, value_kind=kind, seed=11)
    assert d == d2 and inds.tobytes() == i2.tobytes() and vals.tobytes() == v2.tobytes()
    N, nnz = inds.shape
    for m in range(N):
        assert inds[m].max() < d[m] and len(np.unique(inds[m])) == d[m]
    keys = np.zeros(nnz, dtype=np.uint64)
    for m in range(N):
        keys = keys * np.uint64(dims[m]) + inds[m]
    assert len(np.unique(keys)) == nnz
    raw, rv, _ = O.generate(dims, 300_000, alpha=alpha, value_kind=kind, seed=11, clean=False)
    assert raw.shape == (N, 300_000) and abs(rv.sum() - vals.sum()) < 1e-9 * abs(rv.sum())
    if alpha:
        assert np.mean(raw[0] == 0) > 5 * np.mean(raw[0] == 50)
    if kind == 1:
        assert rv.min() > 0 and abs(np.mean(np.log(rv))) < 0.01
    else:
        assert rv.min() >= 0 and rv.max() < 1
