"""SPACE_EFFICIENT plans (trees only for the groups that memoize, tag-2
recompute for the rest): the host decision against the reference's own
decide_use_csfs (oracle/_ref) and the oracle restatement, then the MTTKRP
sequence and ALS on the GPU."""
import ctypes as C
import itertools

import numpy as np
import pytest

import adatm_b200 as A
import oracle as O
from _gen import dense_mttkrp
from conftest import load_golden

SENTINEL = 99


def _ref_decide(N, groups, n_csf):
    """The reference's decide_use_csfs (compiled from its mttkrp.c)."""
    from adatm_b200._native import GroupProperties
    L = O.ref()
    oo = [np.ascontiguousarray(g["o_opt"], dtype=np.uint64) for g in groups]
    arr = (GroupProperties * len(groups))()
    for i, g in enumerate(groups):
        arr[i].memo_mode = g["memo_mode"]
        arr[i].begin_imten = g["begin_imten"]
        arr[i].n_imten = g["n_imten"]
        arr[i].o_opt = oo[i].ctypes.data_as(C.POINTER(C.c_uint64))
    uc = np.full(N, SENTINEL, dtype=np.uint64)
    ut = np.full(N, SENTINEL, dtype=np.uint64)
    L.decide_use_csfs.argtypes = [C.c_uint64, C.POINTER(GroupProperties), C.c_int, C.c_uint64,
                                  C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.decide_use_csfs.restype = None
    L.decide_use_csfs(N, arr, len(groups), n_csf, uc.ctypes.data_as(C.POINTER(C.c_uint64)),
                      ut.ctypes.data_as(C.POINTER(C.c_uint64)))
    return uc, ut


def _space_cases():
    cases = []
    for N in range(4, 9):
        for memo_modes in itertools.combinations(range(N - 1), 3 if N >= 6 else 2):
            if memo_modes[0] != 0:
                continue
            for mask in range(1, 2 ** len(memo_modes) - 1):
                groups = []
                for k, mm in enumerate(memo_modes):
                    memo = (mask >> k) & 1
                    nxt = memo_modes[k + 1] if k + 1 < len(memo_modes) else N
                    n_imten = min(nxt - mm - 1, N - 2 - 0) if memo else 0
                    groups.append({"memo_mode": mm, "begin_imten": max(1, n_imten) if memo else 1,
                                   "n_imten": max(0, n_imten) if memo else 0,
                                   "o_opt": [mm] + [m for m in range(N) if m != mm]})
                if all(g["n_imten"] == 0 for g in groups):
                    continue
                cases.append((N, groups))
    return cases


@pytest.mark.skipif(not O.ref_available(), reason="the reference's code is not built here")
def test_space_branch_matches_reference_code():
    checked = 0
    for N, groups in _space_cases():
        n_csf = sum(1 for g in groups if g["n_imten"] > 0)
        if n_csf == len(groups):
            continue
        ruc, rut = _ref_decide(N, groups, n_csf)
        uc, ut = A.decide_use_csfs(N, groups, n_csf)
        ouc, out_ = O.decide_use_csfs(N, groups, n_csf)
        for m in range(N):
            if ruc[m] == SENTINEL:  # left unassigned by the reference: recompute on tree 0
                assert (uc[m], ut[m]) == (0, 2)
            else:
                assert (uc[m], ut[m]) == (ruc[m], rut[m]), (N, groups, m)
                assert (ouc[m], out_[m]) == (ruc[m], rut[m])
        checked += 1
    assert checked > 20


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["n5_zipf", "n6_uniform", "n8_uniform"])
def test_space_efficient_sequence_and_als(gpu, name):
    d = load_golden(name)
    N, R = d["N"], int(d["R"])
    groups = [dict(g) for g in d["groups"]]
    if len(groups) < 2:
        pytest.skip("one group: SPACE_EFFICIENT is the TIME_EFFICIENT plan")
    groups[-1] = dict(groups[-1], n_imten=0)  # the last group recomputes
    if all(g["n_imten"] == 0 for g in groups):
        pytest.skip("no memoizing group left")
    opts = A.splatt_default_opts()
    opts[A.OPT_CSF_ALLOC] = A.ADAPTIVE_SPACE_EFFICIENT
    cs = A.csf_alloc_adaptive(d["inds"], d["vals"], d["dims_list"], groups, opts)
    n_memo = sum(1 for g in groups if g["n_imten"] > 0)
    assert len(cs) == n_memo
    rs = A.rcsf_alloc_adaptive(cs, R, groups, opts)
    uc, ut = A.decide_use_csfs(N, groups, len(cs))
    assert 2 in set(ut.tolist())
    mats = O.init_factors(d["dims_list"], R, 0)
    for _ in range(2):
        for m in range(N):
            out = A.mttkrp_csf_adaptive(cs, rs, mats, m, groups, uc, ut, opts)
            ref = dense_mttkrp(d["inds"], d["vals"], d["dims_list"], mats, m)
            assert np.max(np.abs(out - ref)) / np.max(np.abs(ref)) < 2e-5
    res = A.cpd_als_iterate_adaptive(cs, rs, groups, uc, ut, mats, 5, 0.0, opts)
    assert abs(res["fit"] - float(d["als5_fit"])) < 1e-4
    cs.free()
