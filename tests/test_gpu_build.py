"""GPU construction (radix sort + level scans) is bit-exact with the oracle,
which is pinned to the reference's own p_csf_alloc_untiled."""
import numpy as np
import pytest

import oracle as O
from conftest import golden_cases, load_golden
from _gen import draw_coo

pytestmark = pytest.mark.gpu


def assert_tree_equal(got, ref, N):
    np.testing.assert_array_equal(got["nfibs"], ref["nfibs"])
    for l in range(N - 1):
        np.testing.assert_array_equal(got["fptr"][l], ref["fptr"][l])
    for l in range(1, N):
        np.testing.assert_array_equal(got["fids"][l], ref["fids"][l])
    assert got["vals"].tobytes() == ref["vals"].tobytes()


@pytest.mark.parametrize("name", golden_cases())
def test_trees_bit_exact_golden(gpu, name):
    d = load_golden(name)
    A = gpu
    t = A.Tensor.from_coo(d["inds"], d["vals"], d["dims_list"])
    plan = {"nmodes": d["N"], "groups": d["groups"]}
    e = A.Engine(t, int(d["R"]), plan)
    for g in range(len(d["groups"])):
        got = e.csf_arrays(g)
        ref = {"nfibs": d[f"g{g}_nfibs"], "vals": d[f"g{g}_vals"],
               "fptr": [d.get(f"g{g}_fptr{l}") for l in range(d["N"])],
               "fids": [None] + [d[f"g{g}_fids{l}"] for l in range(1, d["N"])]}
        assert_tree_equal(got, ref, d["N"])
        # fids[0] holds the root ids; after compaction they are 0..F0-1
        np.testing.assert_array_equal(got["fids"][0], np.arange(int(d[f"g{g}_nfibs"][0])))


@pytest.mark.parametrize("dims,nnz,alpha,seed", [
    ([1000, 1000, 1000], 200000, None, 0),
    ([5000, 5000, 2000, 500], 300000, 1.1, 1),
    ([20000, 10000, 5000, 1000, 200], 300000, 1.2, 2),
    ([50000, 20000, 10000, 2000, 500, 100], 200000, 1.3, 3),       # 72-bit keys (two words)
    ([100000, 90000, 80000, 70000, 60000, 50000, 40000, 30000], 50000, 1.0, 4),  # three words
    ([2, 3, 2], 10, None, 5),
])
def test_trees_bit_exact_random(gpu, dims, nnz, alpha, seed):
    A = gpu
    inds, vals, dims = draw_coo(dims, nnz, seed, alpha)
    ci, cv, cd = O.coo_clean(inds, vals, dims)
    cd = [int(x) for x in cd]
    t = A.Tensor.from_coo(ci, cv, cd)
    rng = np.random.default_rng(seed)
    N = len(cd)
    for trial in range(2):
        perm = list(rng.permutation(N))
        plan = {"nmodes": N, "groups": [{"memo_mode": perm[0], "begin_imten": 1, "n_imten": 0,
                                         "o_opt": perm}],
                "use_csfs": [0] * N, "use_tags": [0 if m == perm[0] else 2 for m in range(N)]}
        e = A.Engine(t, 4, plan)
        ref = O.csf_build(ci, cv, cd, perm)
        assert_tree_equal(e.csf_arrays(0), ref, N)
        np.testing.assert_array_equal(t.count_nfibs(perm), ref["nfibs"])


def test_duplicates_kept_as_leaves_like_reference(gpu):
    """Without cleaning, duplicate coordinates stay separate leaves in input
    order (stable sort), as the reference's construction keeps them."""
    A = gpu
    inds = np.array([[1, 0, 1, 1], [2, 0, 2, 2], [0, 1, 0, 0]], dtype=np.uint64)
    vals = np.array([1.0, 2.0, 3.0, 4.0])
    t = A.Tensor.from_coo(inds, vals, [2, 3, 2])
    plan = {"nmodes": 3, "groups": [{"memo_mode": 0, "begin_imten": 1, "n_imten": 0, "o_opt": [0, 1, 2]}],
            "use_csfs": [0, 0, 0], "use_tags": [0, 2, 2]}
    got = A.Engine(t, 2, plan).csf_arrays(0)
    ref = O.csf_build(inds, vals, [2, 3, 2], [0, 1, 2])
    assert_tree_equal(got, ref, 3)
    assert got["vals"].tolist() == [2.0, 1.0, 3.0, 4.0]


@pytest.mark.parametrize("dims,nnz,alpha,seed", [([40, 30, 20, 10], 20000, 1.4, 7),
                                                 ([300, 200, 100], 50000, None, 8)])
def test_coo_clean_matches_oracle(gpu, dims, nnz, alpha, seed):
    A = gpu
    inds, vals, dims = draw_coo(dims, nnz, seed, alpha)
    t = A.Tensor.from_coo(inds, vals, dims, clean=True)
    gi, gv, gd = t.download()
    ci, cv, cd = O.coo_clean(inds, vals, dims)
    assert gd == [int(x) for x in cd]
    np.testing.assert_array_equal(gi, ci)
    assert gv.tobytes() == cv.tobytes()


def test_generator_is_deterministic_and_clean(gpu):
    A = gpu
    a = A.Tensor.generate([500, 400, 300, 200], 100000, alpha=1.1, seed=3)
    b = A.Tensor.generate([500, 400, 300, 200], 100000, alpha=1.1, seed=3)
    ia, va, da = a.download()
    ib, vb, db = b.download()
    np.testing.assert_array_equal(ia, ib)
    assert va.tobytes() == vb.tobytes() and da == db
    # cleaned: unique coordinates, every slice of every mode used
    keys = {tuple(c) for c in ia.T.tolist()}
    assert len(keys) == ia.shape[1]
    for m in range(4):
        assert set(ia[m].tolist()) == set(range(da[m]))
    # Zipf(1.1): index 0 is the most frequent in every mode
    for m in range(4):
        counts = np.bincount(ia[m].astype(np.int64))
        assert counts.argmax() == 0


def test_bad_inputs_rejected(gpu):
    A = gpu
    with pytest.raises(A.AdatmError) as ei:
        A.Tensor.from_coo(np.array([[5], [0], [0]], dtype=np.uint64), [1.0], [3, 3, 3])
    assert ei.value.code == A.SPLATT_ERROR_BADINPUT
    with pytest.raises(A.AdatmError):
        A.Tensor.from_coo(np.zeros((2, 3), dtype=np.uint64), [1.0, 2.0, 3.0], [3, 3])


def test_empty_tensor(gpu):
    A = gpu
    t = A.Tensor.from_coo(np.zeros((3, 0), dtype=np.uint64), np.zeros(0), [2, 2, 2])
    assert list(t.count_nfibs([0, 1, 2])) == [0, 0, 0]
