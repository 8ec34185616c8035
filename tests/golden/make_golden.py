"""Generate the golden fixtures from the reference's own AdaTM code.

The reference ships no tests or golden vectors, so these fixtures are made by
running its own C files (adatm_rcsf.c, mttkrp.c, adatm_bench.c, adatm_cpd.c,
adatm_utils.c, adatm_sort.c compiled into oracle/_ref/libadatm_ref.so against
the SPLATT stand-in in oracle/shim) on small seeded tensors:

* the plan decide_parameters_auto picks (N >= 4; for N = 3 the reference's
  candidate count is undefined and the fixture stores the single candidate);
* the arrays of every CSF csf_alloc_adaptive builds;
* use_csfs / use_tags of decide_use_csfs;
* every mode's mttkrp_csf_adaptive output over two MTTKRP sequences (memo
  buffers zeroed before each memo-root call, one thread);
* cpd_als_iterate_adaptive's fit and lambda after 5 iterations.

Run from the repository root where the reference checkout exists:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle as O  # noqa: E402
from _gen import draw_coo  # noqa: E402

CASES = [
    dict(name="n3_uniform", dims=[30, 40, 50], nnz=3000, R=8, seed=1, alpha=None),
    dict(name="n4_zipf", dims=[40, 35, 25, 20], nnz=5000, R=8, seed=2, alpha=1.1),
    dict(name="n4_ties", dims=[20, 20, 20, 20], nnz=3000, R=6, seed=5, alpha=None),
    dict(name="n5_zipf", dims=[14, 12, 10, 9, 8], nnz=4000, R=8, seed=3, alpha=1.2),
    dict(name="n6_uniform", dims=[6, 7, 5, 8, 6, 7], nnz=3000, R=4, seed=4, alpha=None),
    dict(name="n7_uniform", dims=[5, 6, 4, 5, 6, 4, 5], nnz=2500, R=4, seed=6, alpha=None),
    dict(name="n8_uniform", dims=[4, 5, 4, 3, 5, 4, 3, 4], nnz=2000, R=4, seed=7, alpha=None),
]


def make(case):
    inds, vals, dims = draw_coo(case["dims"], case["nnz"], case["seed"], case["alpha"])
    inds, vals, dims = O.coo_clean(inds, vals, dims)
    dims = [int(d) for d in dims]
    N = len(dims)
    R = case["R"]
    groups = O.ref_plan(inds, vals, dims, R)
    if groups is None:
        groups, _ = O.plan(inds, dims, R)
    rm = O.RefModel(inds, vals, dims, R, groups, nthreads=1)
    uc, ut = rm.use()
    out = {"inds": inds, "vals": vals, "dims": np.array(dims, dtype=np.uint64),
           "R": np.array(R), "n_grp": np.array(len(groups)),
           "use_csfs": uc, "use_tags": ut}
    for g, gr in enumerate(groups):
        out[f"g{g}_memo_mode"] = np.array(gr["memo_mode"])
        out[f"g{g}_begin_imten"] = np.array(gr["begin_imten"])
        out[f"g{g}_n_imten"] = np.array(gr["n_imten"])
        out[f"g{g}_o_opt"] = np.array(gr["o_opt"], dtype=np.uint64)
        c = rm.csf(g)
        out[f"g{g}_nfibs"] = c["nfibs"]
        out[f"g{g}_vals"] = c["vals"]
        for l in range(N):
            if c["fptr"][l] is not None:
                out[f"g{g}_fptr{l}"] = c["fptr"][l]
            if c["fids"][l] is not None:
                out[f"g{g}_fids{l}"] = c["fids"][l]
    mats = O.init_factors(dims, R, 0)
    for it in range(2):
        for m in range(N):
            out[f"mttkrp_it{it}_m{m}"] = rm.mttkrp(mats, m)
    res = rm.cpd_als(mats, 5, 0.0)
    out["als5_fit"] = np.array(res["fit"])
    out["als5_lambda"] = res["lambda"]
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                     case["name"] + ".npz"), **out)
    return groups


if __name__ == "__main__":
    if not O.ref_available():
        O.build()
    for c in CASES:
        g = make(c)
        print(c["name"], g)
