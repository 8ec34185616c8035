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
