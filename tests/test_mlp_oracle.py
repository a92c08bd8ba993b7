"""The cost model's CPU oracle: its analytic gradient agrees with central
finite differences (float64)."""
import numpy as np

from oracle import mlp_ref


def test_analytic_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.3, mlp_ref.NP)
    X = rng.normal(0, 1, (40, 16))
    y = rng.normal(0, 1, 40)
    g = mlp_ref.grad(p, X, y)
    idx = np.concatenate([rng.integers(0, mlp_ref.NP, 60), [mlp_ref.NP - 1]])
    fd = mlp_ref.fd_grad(p, X, y, idx)
    assert np.allclose(g[idx], fd, rtol=1e-5, atol=1e-7)
