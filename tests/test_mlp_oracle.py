"""The numpy network oracle against finite differences (CPU)."""

import numpy as np

from oracle import mlp_oracle


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    dims = mlp_oracle.layer_dims(5, 2, 16, 3)
    count = sum(a * b + b for a, b in zip(dims[:-1], dims[1:]))
    params = rng.standard_normal(count) * 0.3
    x = rng.standard_normal((7, 5))
    y = rng.standard_normal((7, 2))
    loss, grad = mlp_oracle.loss_and_gradients(params, dims, x, y)
    assert grad.shape == params.shape and loss > 0
    h = 1e-6
    for index in rng.choice(count, 40, replace=False):
        e = np.zeros(count)
        e[index] = h
        plus, _ = mlp_oracle.loss_and_gradients(params + e, dims, x, y)
        minus, _ = mlp_oracle.loss_and_gradients(params - e, dims, x, y)
        assert abs((plus - minus) / (2 * h) - grad[index]) <= 1e-6 * max(1.0, abs(grad[index]))


def test_oracle_layout_and_forward():
    dims = mlp_oracle.layer_dims(2, 1, 3, 1)
    # W0 (2x3), b0 (3), W1 (3x1), b1 (1)
    params = np.array([1, 0, -1, 0, 1, 1, 0.5, -0.5, 0.0, 1, 2, 3, 0.25], float)
    out = mlp_oracle.forward(params, dims, np.array([[1.0, 2.0]]))[-1]
    hidden = np.maximum(np.array([1.0, 2.0]) @ params[:6].reshape(2, 3) + params[6:9], 0.0)
    assert np.allclose(out, hidden @ params[9:12].reshape(3, 1) + params[12])
