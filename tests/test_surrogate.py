"""The surrogate network's CPU oracle (FP64) against finite differences, and its layout."""
import numpy as np

import mlp as oracle_mlp


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    dims = [7, 5, 5, 1]
    n_params = sum(i * o + o for i, o in zip(dims[:-1], dims[1:]))
    params = rng.normal(0, 0.5, n_params)
    x = rng.normal(0, 1, (11, dims[0]))
    y = (rng.uniform(size=11) < 0.3).astype(float)
    loss, grad = oracle_mlp.loss_and_gradients(params, dims, x, y)
    eps = 1e-6
    for k in rng.choice(n_params, 25, replace=False):
        p = params.copy()
        p[k] += eps
        up, _ = oracle_mlp.loss_and_gradients(p, dims, x, y)
        p[k] -= 2 * eps
        down, _ = oracle_mlp.loss_and_gradients(p, dims, x, y)
        assert abs((up - down) / (2 * eps) - grad[k]) < 1e-7 * max(1.0, abs(grad[k]))
    assert loss > 0
