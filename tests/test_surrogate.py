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


def test_judge_reverts_on_rate_error_not_on_counting_noise():
    from mind_b200.surrogate import judge_populations

    # 100 surrogate and 2 sample cells per population, 1 s observed
    sur_cells, det_cells = np.array([100.0] * 4), np.array([2.0] * 4)
    det = np.array([20.0, 20.0, 2.0, 20.0])            # 10 Hz samples (1 Hz in population 2)
    sur = np.array([1000.0, 3000.0, 200.0, 1040.0])    # 10, 30, 2, 10.4 Hz
    revert = judge_populations(sur, sur_cells, det, det_cells, 1.0, bound=0.05, z=3.0)
    # population 1 fires 3x its sample: reverted; population 3 is 4% off: kept; population 2
    # is 2x off but its sample saw 2 spikes: within the counting noise
    assert revert.tolist() == [False, True, False, False]
    # populations without surrogate cells or without a sample are not judged
    assert not judge_populations([5.0], [0.0], [50.0], [2.0], 1.0, 0.05).any()
    assert not judge_populations([500.0], [100.0], [0.0], [0.0], 1.0, 0.05).any()
