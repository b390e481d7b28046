"""The controller network's CUDA forward/backward/Adam kernels against the
FP64 numpy restatement (oracle/mlp_oracle.py)."""
import numpy as np
import pytest

import dsgdpp_b200 as P
from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


def _net(seed=3):
    net = P.Mlp(seed=seed)
    rng = np.random.default_rng(seed)
    net.params = rng.normal(0, 0.15, net.n_params).astype(np.float32)
    return net, rng


def test_forward_matches_oracle():
    net, rng = _net()
    X = rng.normal(0, 1.5, (40, 16)).astype(np.float32)
    got = net.forward(X)
    want, _ = M.forward(net.params, X)
    np.testing.assert_allclose(got, want, rtol=1e-4, atol=1e-5)
    assert np.all(np.abs(got) <= 1.0)


def test_gradient_matches_oracle():
    net, rng = _net(5)
    X = rng.normal(0, 1.0, (64, 16)).astype(np.float32)
    y = rng.uniform(-0.9, 0.9, 64).astype(np.float32)
    loss, g = net.gradient(X, y)
    wl, wg = M.loss_and_grad(net.params, X, y)
    assert loss == pytest.approx(wl, rel=1e-4)
    scale = np.max(np.abs(wg))
    np.testing.assert_allclose(g, wg, rtol=2e-3, atol=2e-5 * scale)
    # deterministic reduction: the same call gives the same bits
    _, g2 = net.gradient(X, y)
    assert np.array_equal(g, g2)


def test_training_reduces_loss():
    net = P.Mlp(seed=11)
    rng = np.random.default_rng(2)
    X = rng.normal(0, 1, (512, 16)).astype(np.float32)
    y = (0.6 * np.tanh(X[:, 0] - 0.5 * X[:, 3])).astype(np.float32)
    first = net.train_step(X, y, lr=3e-3)
    for _ in range(300):
        last = net.train_step(X, y, lr=3e-3)
    assert last < 0.2 * first
