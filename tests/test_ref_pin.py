"""The oracle restatement against the reference's own code on fresh random
inputs (runs where oracle/_ref was built)."""
import numpy as np
import pytest

import oracle as O
from _gen import draw_coo

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built here")


@pytest.mark.parametrize("seed,dims,alpha", [(11, [15, 20, 9, 12], 1.3), (12, [8, 9, 10, 7, 6], None),
                                             (13, [6, 6, 6, 6, 6, 6], 1.0), (14, [12, 12, 12, 12], None)])
def test_oracle_equals_reference_code(seed, dims, alpha):
    inds, vals, dims = draw_coo(dims, 2500, seed, alpha)
    inds, vals, dims = O.coo_clean(inds, vals, dims)
    dims = [int(x) for x in dims]
    R = 6
    rg = O.ref_plan(inds, vals, dims, R)
    og, _ = O.plan(inds, dims, R)
    assert rg == og
    rm = O.RefModel(inds, vals, dims, R, og)
    om = O.Model(inds, vals, dims, R, og)
    mats = O.init_factors(dims, R, seed)
    for m in range(len(dims)):
        np.testing.assert_array_equal(om.mttkrp(mats, m), rm.mttkrp(mats, m))
    assert abs(om.cpd_als(mats, 4, 0.0)["fit"] - rm.cpd_als(mats, 4, 0.0)["fit"]) < 1e-13
