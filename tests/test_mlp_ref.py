"""The numpy reference network used to check the GPU kernels: its gradient
against central finite differences (CPU only)."""
import numpy as np

from _mlp_ref import loss_and_grad


def test_reference_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    widths = [5, 7, 6, 1]
    n = sum(widths[l + 1] * widths[l] + widths[l + 1] for l in range(len(widths) - 1))
    p = rng.normal(size=n) * 0.5
    X = rng.normal(size=(11, 5))
    T = rng.normal(size=11)
    _, g = loss_and_grad(p, widths, X, T)
    h = 1e-6
    fd = np.zeros(n)
    for k in range(n):
        e = np.zeros(n)
        e[k] = h
        fd[k] = (loss_and_grad(p + e, widths, X, T)[0] - loss_and_grad(p - e, widths, X, T)[0]) / (2 * h)
    np.testing.assert_allclose(g, fd, rtol=1e-5, atol=1e-8)
