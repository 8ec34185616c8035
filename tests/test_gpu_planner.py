"""The learned plan model on the GPU: forward and gradient kernels against the
FP64 numpy reference, Adam training, candidate features and the learned plan
through the C ABI."""
import numpy as np
import pytest

from _mlp_ref import forward as ref_forward
from _mlp_ref import loss_and_grad

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("widths,B", [([16, 64, 64, 1], 300), ([5, 7, 1], 17), ([3, 1], 4),
                                      ([16, 32, 32, 32, 1], 1000)])
def test_forward_and_gradient_match_reference(gpu, widths, B):
    A = gpu
    net = A.Mlp(widths, seed=3)
    p = net.get_params()
    rng = np.random.default_rng(B)
    X = rng.normal(size=(B, widths[0])).astype(np.float32)
    T = rng.normal(size=B).astype(np.float32)
    y = net.forward(X)
    yr, _, _ = ref_forward(p, widths, X)
    np.testing.assert_allclose(y, yr, rtol=1e-4, atol=1e-5 * max(1.0, np.abs(yr).max()))
    loss, g = net.gradient(X, T)
    lr, gr = loss_and_grad(p, widths, X, T)
    assert abs(loss - lr) <= 1e-4 * max(1.0, lr)
    assert np.max(np.abs(g - gr)) <= 1e-4 * max(1e-3, np.max(np.abs(gr)))


def test_adam_training_fits_a_smooth_target(gpu):
    A = gpu
    rng = np.random.default_rng(0)
    X = rng.uniform(-1, 1, size=(2048, 6)).astype(np.float32)
    T = (np.sin(2 * X[:, 0]) + X[:, 1] * X[:, 2] + 0.5 * X[:, 3] ** 2).astype(np.float32)
    net = A.Mlp([6, 32, 32, 1], seed=1)
    before, _ = net.gradient(X, T)
    after = net.train(X, T, epochs=200, batch=128, lr=3e-3, seed=0)
    final, _ = net.gradient(X, T)
    assert final < 0.05 * before and final < 0.01, (before, after, final)
    # seeded: the same schedule gives the same parameters
    net2 = A.Mlp([6, 32, 32, 1], seed=1)
    net2.train(X, T, epochs=200, batch=128, lr=3e-3, seed=0)
    np.testing.assert_array_equal(net.get_params(), net2.get_params())


def test_plan_features_and_learned_plan(gpu):
    A = gpu
    t = A.Tensor.generate([300, 200, 150, 100, 80], 200_000, alpha=1.2, seed=5)
    X, nbytes, cands = A.plan_features(t, 16)
    plan, acands, chosen = A.plan_analytic(t, 16)
    assert X.shape == (len(acands), A.PLAN_FEATURES) and np.all(np.isfinite(X))
    assert [c["groups"] for c in cands] == [c["groups"] for c in acands]
    assert np.all(nbytes > 0)
    # no model: the analytic plan
    p0, c0, used = A.plan_learned(t, 16, None)
    assert not used and c0 == chosen and p0["groups"] == plan["groups"]
    # a model that scores candidates by one feature picks that feature's minimum
    widths = [A.PLAN_FEATURES, 1]
    params = np.zeros(A.PLAN_FEATURES + 1, dtype=np.float32)
    params[14] = 1.0  # total tree nodes per nonzero
    model = A.PlanModel(widths, params, np.zeros(A.PLAN_FEATURES), np.ones(A.PLAN_FEATURES))
    p1, c1, used = A.plan_learned(t, 16, model)
    assert used and c1 == int(np.argmin(X[:, 14]))
    e = A.Engine(t, 16, p1)
    e.init_factors(0)
    r1 = e.als(3, 0.0)
    e0 = A.Engine(t, 16, p0)
    e0.init_factors(0)
    r0 = e0.als(3, 0.0)
    assert abs(r1["fit"] - r0["fit"]) < 1e-4


def test_committed_model_through_the_library(gpu):
    """The shipped model loaded into the GPU network picks, through
    adatm_plan_learned, the candidate its numpy forward ranks first."""
    import os
    from conftest import ROOT
    from _mlp_ref import forward
    A = gpu
    path = os.path.join(ROOT, "adatm_b200", "planner_data", "plan_model.npz")
    model = A.PlanModel.load(path)
    t = A.Tensor.generate([3000, 1200, 800, 400, 200, 60], 600_000, alpha=1.25, seed=11)
    X, _, _ = A.plan_features(t, 32)
    z = np.load(path)
    pred, _, _ = forward(z["params"], [int(w) for w in z["widths"]], (X - z["mean"]) / z["std"])
    np.testing.assert_allclose(model.predict(X), pred, rtol=1e-4, atol=1e-4)
    plan, chosen, used = A.plan_learned(t, 32, model)
    assert used and chosen == int(np.argmin(pred))
