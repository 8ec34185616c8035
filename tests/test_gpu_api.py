"""The drop-in C ABI: SPLATT's public functions and AdaTM's entry points,
called the way the reference's CLI and bench call them."""
import numpy as np
import pytest

import oracle as O
from conftest import golden_cases, load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", golden_cases())
def test_adatm_entry_point_sequence(gpu, name):
    """decide_parameters_auto -> csf_alloc_adaptive -> rcsf_alloc_adaptive ->
    decide_use_csfs -> mttkrp_csf_adaptive x N x 2, as bench_adaptm runs it."""
    A = gpu
    d = load_golden(name)
    N, R = d["N"], int(d["R"])
    groups = A.decide_parameters_auto(d["inds"], d["vals"], d["dims_list"], R)
    assert groups == d["groups"]
    opts = A.splatt_default_opts()
    cs = A.csf_alloc_adaptive(d["inds"], d["vals"], d["dims_list"], groups, opts)
    assert len(cs) == len(groups)
    for g in range(len(groups)):
        tr = cs.tree(g)
        np.testing.assert_array_equal(tr["nfibs"], d[f"g{g}_nfibs"])
        for l in range(N - 1):
            np.testing.assert_array_equal(tr["fptr"][l], d[f"g{g}_fptr{l}"])
        for l in range(1, N):
            np.testing.assert_array_equal(tr["fids"][l], d[f"g{g}_fids{l}"])
        assert tr["fids"][0] is None
        assert tr["vals"].tobytes() == d[f"g{g}_vals"].tobytes()
    rs = A.rcsf_alloc_adaptive(cs, R, groups, opts)
    uc, ut = A.decide_use_csfs(N, groups, len(cs))
    mats = O.init_factors(d["dims_list"], R, 0)
    for it in range(2):
        for m in range(N):
            out = A.mttkrp_csf_adaptive(cs, rs, mats, m, groups, uc, ut, opts)
            ref = d[f"mttkrp_it{it}_m{m}"]
            assert np.max(np.abs(out - ref)) / np.max(np.abs(ref)) < 2e-5
    # memo trees: reference shapes, device rows pulled to the host views
    rs.pull()
    j = 0
    for g, gr in enumerate(groups):
        if gr["n_imten"] == 0:
            continue
        for deg in range(gr["n_imten"]):
            mm = rs.memo(j, deg)
            assert mm["nmodes"] == gr["begin_imten"] - deg + 1
            assert mm["nnz"] == int(d[f"g{g}_nfibs"][mm["nmodes"] - 2]) * R
            assert np.all(np.isfinite(mm["vals"]))
        j += 1
    res = A.cpd_als_iterate_adaptive(cs, rs, groups, uc, ut, mats, 5, 0.0, opts)
    assert abs(res["fit"] - float(d["als5_fit"])) < 1e-4
    cs.free()


@pytest.mark.parametrize("alloc", [0, 1, 2, 4])
def test_splatt_public_api(gpu, alloc):
    A = gpu
    d = load_golden("n4_zipf")
    opts = A.splatt_default_opts()
    opts[A.OPT_CSF_ALLOC] = alloc
    opts[A.OPT_NITER] = 5
    opts[A.OPT_TOLERANCE] = 0.0
    cs = A.splatt_csf_convert(d["inds"], d["vals"], opts)
    R = 8
    mats = O.init_factors(d["dims_list"], R, 0)
    for m in range(4):
        ref = O.mttkrp_csf(d["inds"], d["vals"], d["dims_list"], O.splatt_perm(d["dims_list"], 1, m),
                           mats, m, R)
        out = A.splatt_mttkrp(m, R, cs, mats, opts)
        assert np.max(np.abs(out - ref)) / np.max(np.abs(ref)) < 2e-5
    k = A.splatt_cpd_als(cs, R, opts)
    assert k["rank"] == R and k["nmodes"] == 4
    if alloc == 4:
        assert abs(k["fit"] - float(d["als5_fit"])) < 1e-4
    for m in range(4):
        np.testing.assert_allclose(np.linalg.norm(k["factors"][m], axis=0), 1.0, rtol=1e-6)
    cs.free()


def _recompute_elsewhere(trees, N):
    """A non-default per-mode (tree, tag) set: each tree's root mode runs its
    root MTTKRP (tag 0); every other mode recomputes (tag 2) on the last tree."""
    roots = {int(t["dim_perm"][0]): g for g, t in enumerate(trees)}
    uc, ut = [], []
    for m in range(N):
        if m in roots:
            uc.append(roots[m])
            ut.append(0)
        else:
            uc.append(len(trees) - 1)
            ut.append(2)
    return uc, ut


@pytest.mark.skipif(not O.ref_available(), reason="the reference's own code (oracle/_ref) is not built")
@pytest.mark.parametrize("name", ["n4_zipf", "n5_zipf", "n6_uniform"])
def test_caller_tags_are_honoured(gpu, name):
    """mttkrp_csf_adaptive and cpd_als_iterate_adaptive run the trees and
    tags the caller passes (use_csfs / use_tags), not the handle's plan: the
    MTTKRP sequence and the 4-iteration fit equal the reference's own
    functions called with the same non-default tags (mttkrp.c:2037-2090,
    adatm_cpd.c:256-373)."""
    A = gpu
    d = load_golden(name)
    N, R = d["N"], int(d["R"])
    groups = d["groups"]
    opts = A.splatt_default_opts()
    cs = A.csf_alloc_adaptive(d["inds"], d["vals"], d["dims_list"], groups, opts)
    rs = A.rcsf_alloc_adaptive(cs, R, groups, opts)
    trees = [cs.tree(g) for g in range(len(cs))]
    ref = O.RefModel(d["inds"], d["vals"], d["dims_list"], R, groups)
    duc, dut = A.decide_use_csfs(N, groups, len(cs))
    duc = [int(x) for x in duc]
    dut = [int(x) for x in dut]
    # (a) recompute on the last tree; (b) memo reuse replaced by recompute
    variants = [_recompute_elsewhere(trees, N), (duc, [2 if t == 1 else t for t in dut])]
    mats = O.init_factors(d["dims_list"], R, 0)
    for uc, ut in variants:
        assert (list(uc), list(ut)) != (duc, dut)
        ref.set_use(uc, ut)
        for m in range(N):
            out = A.mttkrp_csf_adaptive(cs, rs, mats, m, groups, uc, ut, opts)
            want = ref.mttkrp(mats, m)
            assert np.max(np.abs(out - want)) / np.max(np.abs(want)) < 2e-5, (uc, ut, m)
        got = A.cpd_als_iterate_adaptive(cs, rs, groups, uc, ut, mats, 4, 0.0, opts)
        want = ref.cpd_als(mats, 4, 0.0)
        assert abs(got["fit"] - want["fit"]) < 1e-4, (uc, ut)
    # the default plan again on the same handle gives the fixture's fit
    res = A.cpd_als_iterate_adaptive(cs, rs, groups, duc, dut, mats, 5, 0.0, opts)
    assert abs(res["fit"] - float(d["als5_fit"])) < 1e-4
    cs.free()


@pytest.mark.parametrize("name", ["n4_zipf", "n5_zipf"])
def test_caller_plan_mismatch_rejected(gpu, name):
    """Plans the trees cannot run are refused with SPLATT_ERROR_BADINPUT
    (and the reason in adatm_last_error), never run silently."""
    A = gpu
    d = load_golden(name)
    N, R = d["N"], int(d["R"])
    groups = d["groups"]
    opts = A.splatt_default_opts()
    cs = A.csf_alloc_adaptive(d["inds"], d["vals"], d["dims_list"], groups, opts)
    rs = A.rcsf_alloc_adaptive(cs, R, groups, opts)
    duc, dut = A.decide_use_csfs(N, groups, len(cs))
    duc = [int(x) for x in duc]
    dut = [int(x) for x in dut]
    mats = O.init_factors(d["dims_list"], R, 0)
    root0 = int(cs.tree(0)["dim_perm"][0])
    nonroot = int(cs.tree(0)["dim_perm"][1])
    bad = []
    uc, ut = list(duc), list(dut)
    uc[nonroot], ut[nonroot] = 0, 0          # tag 0 on a mode that is not the tree's root
    bad.append((uc, ut, "root"))
    uc, ut = list(duc), list(dut)
    uc[root0], ut[root0] = 0, 2              # tag 2 on a tree's root
    bad.append((uc, ut, "root"))
    uc, ut = list(duc), list(dut)
    uc[nonroot] = len(cs) + 3                # a tree that does not exist
    bad.append((uc, ut, "tree"))
    uc, ut = list(duc), list(dut)
    ut[nonroot] = 7                          # a tag outside 0..2
    bad.append((uc, ut, "use_tags"))
    for uc, ut, word in bad:
        with pytest.raises(A.AdatmError) as e:
            A.cpd_als_iterate_adaptive(cs, rs, groups, uc, ut, mats, 1, 0.0, opts)
        assert e.value.code == A.SPLATT_ERROR_BADINPUT
        assert word in str(e.value)
    # memo reuse with no root MTTKRP of its tree earlier in the sweep: the
    # tree's root mode itself reuses rows nothing has written yet
    if 1 in dut:
        t = duc[dut.index(1)]
        r = int(cs.tree(t)["dim_perm"][0])
        uc, ut = list(duc), list(dut)
        ut[r] = 1
        with pytest.raises(A.AdatmError) as e:
            A.cpd_als_iterate_adaptive(cs, rs, groups, uc, ut, mats, 1, 0.0, opts)
        assert "earlier mode" in str(e.value)
    # groups whose level order is not that of the trees
    g2 = [dict(g, o_opt=list(reversed(g["o_opt"]))) for g in groups]
    with pytest.raises(A.AdatmError) as e:
        A.cpd_als_iterate_adaptive(cs, rs, g2, duc, dut, mats, 1, 0.0, opts)
    assert "o_opt" in str(e.value)
    # a single MTTKRP with a tag the tree cannot run
    with pytest.raises(A.AdatmError):
        A.mttkrp_csf_adaptive(cs, rs, mats, nonroot, groups, [0] * N, [0] * N, opts)
    # the handle still works with the default plan afterwards
    res = A.cpd_als_iterate_adaptive(cs, rs, groups, duc, dut, mats, 5, 0.0, opts)
    assert abs(res["fit"] - float(d["als5_fit"])) < 1e-4
    cs.free()


def test_overlapped_download_is_the_plain_download(gpu):
    """cpd_als_iterate_adaptive copies the last sweep's factors out mode by
    mode while the sweep runs. Two sweeps that way must give the factors,
    lambda and fit of three allowed sweeps stopped by the tolerance after two
    (whose factors come back after the sweep), bit for bit."""
    A = gpu
    name = golden_cases()[0]
    d = load_golden(name)
    N, R = d["N"], int(d["R"])
    groups = A.decide_parameters_auto(d["inds"], d["vals"], d["dims_list"], R)
    cs = A.csf_alloc_adaptive(d["inds"], d["vals"], d["dims_list"], groups)
    rs = A.rcsf_alloc_adaptive(cs, R, groups)
    uc, ut = A.decide_use_csfs(N, groups, len(cs))
    mats = O.init_factors(d["dims_list"], R, 2)
    a = A.CpdIterator(cs, rs, groups, uc, ut, mats)
    fa = a.step(2, 0.0)
    b = A.CpdIterator(cs, rs, groups, uc, ut, mats)
    fb = b.step(3, 1e9)
    assert fa == fb
    for m in range(N):
        assert a.factors[m].tobytes() == b.factors[m].tobytes(), m
    assert a.lam.tobytes() == b.lam.tobytes()
    cs.free()
