"""The FP64 MLP oracle against finite differences (pins the gradient checks
of the CUDA training kernels)."""
import numpy as np

from oracle import mlp


def test_param_count():
    assert mlp.N_PARAMS == 5187


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = mlp.init(1) + rng.normal(0, 0.05, mlp.N_PARAMS)
    x = rng.normal(0, 1, (37, 12))
    t = rng.normal(0, 1, (37, 3))
    loss, g = mlp.loss_and_grad(p, x, t)
    idx = rng.choice(mlp.N_PARAMS, 60, replace=False)
    eps = 1e-6
    for q in idx:
        e = np.zeros_like(p)
        e[q] = eps
        lp, _ = mlp.loss_and_grad(p + e, x, t)
        lm, _ = mlp.loss_and_grad(p - e, x, t)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[q]) <= 1e-6 * max(1.0, abs(fd)), (q, fd, g[q])


def test_gelu_grad():
    x = np.linspace(-5, 5, 101)
    fd = (mlp.gelu(x + 1e-6) - mlp.gelu(x - 1e-6)) / 2e-6
    assert np.allclose(mlp.gelu_grad(x), fd, atol=1e-7)
