"""The numpy restatement of the controller MLP that checks the device kernels:
its analytic gradient against central finite differences."""
import numpy as np

from .mlp_ref import forward, loss_and_grad


def test_reference_gradient_matches_finite_differences():
    n_in, h, n_out = 5, 7, 2
    rng = np.random.default_rng(0)
    n_p = h * n_in + h + h * h + h + n_out * h + n_out
    p = rng.normal(scale=0.4, size=n_p)
    x = rng.normal(size=(9, n_in))
    t = rng.normal(size=(9, n_out))
    _, g = loss_and_grad(p, x, t, n_in, h, n_out)
    eps = 1e-6
    fd = np.empty(n_p)
    for q in range(n_p):
        e = np.zeros(n_p)
        e[q] = eps
        fd[q] = (loss_and_grad(p + e, x, t, n_in, h, n_out)[0] - loss_and_grad(p - e, x, t, n_in, h, n_out)[0]) / (2 * eps)
    assert np.max(np.abs(fd - g)) < 1e-7 * max(1.0, np.max(np.abs(g)))
    y, _ = forward(p, x, n_in, h, n_out)
    assert y.shape == (9, n_out)
