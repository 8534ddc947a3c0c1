"""The chooser's network: the numpy oracle checked by finite differences (CPU), the GPU
kernels' loss, gradients and predictions checked against the oracle, and GPU training."""
import numpy as np
import pytest

from oracle.mlp_oracle import forward, loss_grad

SHAPE = (7, 16, 5)


def _data(seed, n=40):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, SHAPE[0])).astype(np.float32)
    T = rng.normal(size=(n, SHAPE[2])).astype(np.float32)
    M = (rng.random((n, SHAPE[2])) > 0.2).astype(np.float32)
    return X, T, M


def _params(seed):
    rng = np.random.default_rng(seed)
    n = SHAPE[0] * SHAPE[1] + SHAPE[1] + SHAPE[1] * SHAPE[1] + SHAPE[1] + SHAPE[1] * SHAPE[2] + SHAPE[2]
    return (rng.normal(size=n) * 0.3).astype(np.float64)


def test_oracle_gradient_matches_finite_differences():
    X, T, M = _data(1)
    p = _params(2)
    loss, g = loss_grad(p, X, T, M, *SHAPE)
    eps = 1e-6
    rng = np.random.default_rng(3)
    for i in rng.choice(p.size, 40, replace=False):
        q = p.copy()
        q[i] += eps
        lp, _ = loss_grad(q, X, T, M, *SHAPE)
        q[i] -= 2 * eps
        lm, _ = loss_grad(q, X, T, M, *SHAPE)
        assert abs((lp - lm) / (2 * eps) - g[i]) < 1e-5 * max(1.0, abs(g[i]))


@pytest.mark.gpu
def test_gpu_loss_and_gradients_match_oracle():
    from vldb_voila_b200.engine import Mlp
    X, T, M = _data(4)
    net = Mlp(*SHAPE, seed=5)
    p = _params(6).astype(np.float32)
    net.set_params(p)
    loss, g = net.loss_grad(X, T, M)
    loss_ref, g_ref = loss_grad(p.astype(np.float64), X, T, M, *SHAPE)
    assert abs(loss - loss_ref) <= 1e-5 * max(1.0, abs(loss_ref))
    np.testing.assert_allclose(g, g_ref, rtol=1e-4, atol=1e-5)
    Y_ref, _ = forward(p.astype(np.float64), X, *SHAPE)
    np.testing.assert_allclose(net.predict(X), Y_ref, rtol=1e-4, atol=1e-5)


@pytest.mark.gpu
def test_gpu_training_fits_a_smooth_target():
    from vldb_voila_b200.engine import Mlp
    rng = np.random.default_rng(8)
    X = rng.uniform(-1, 1, size=(512, SHAPE[0])).astype(np.float32)
    T = np.stack([np.sin(2 * X[:, 0]) + X[:, 1] * X[:, 2], X[:, 3] ** 2, np.abs(X[:, 4]), X[:, 5] - X[:, 6],
                  np.cos(X[:, 0] + X[:, 1])], axis=1).astype(np.float32)
    net = Mlp(*SHAPE, seed=9)
    l0, _ = net.loss_grad(X, T)
    l1 = net.train(X, T, epochs=300, batch=64, lr=3e-3, seed=10)
    assert l1 < l0 / 10
    # deterministic: same seed, same data -> same parameters
    net2 = Mlp(*SHAPE, seed=9)
    net2.train(X, T, epochs=300, batch=64, lr=3e-3, seed=10)
    np.testing.assert_array_equal(net.get_params(), net2.get_params())
