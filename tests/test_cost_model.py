"""The cost model's network: device gradients and predictions against the
float64 NumPy restatement, and the restatement against finite differences."""

import numpy as np
import pytest

import mlp_oracle


def _params(seed=0):
    rng = np.random.default_rng(seed)
    w = np.empty(64 * 24 + 64 + 64 * 64 + 64 + 64 + 1)
    o = 0
    for n, fan in ((64 * 24, 24), (64, 0), (64 * 64, 64), (64, 0), (64, 64), (1, 0)):
        w[o:o + n] = rng.normal(0, np.sqrt(2 / fan), n) if fan else rng.normal(0, 0.1, n)
        o += n
    return w.astype(np.float32)


def _data(n, seed=1):
    rng = np.random.default_rng(seed)
    X = rng.normal(0, 1, (n, 24)).astype(np.float32)
    y = (X[:, 0] * 0.7 - np.abs(X[:, 1]) + 0.3 * X[:, 2] * X[:, 3]).astype(np.float32)
    return X, y


def test_oracle_gradient_matches_finite_differences():
    w = _params().astype(np.float64)
    X, y = _data(40)
    _, g = mlp_oracle.loss_grad(w, X, y)
    rng = np.random.default_rng(5)
    for k in rng.choice(len(w), 60, replace=False):
        e = np.zeros_like(w)
        e[k] = 1e-6
        fd = (mlp_oracle.loss_grad(w + e, X, y)[0] - mlp_oracle.loss_grad(w - e, X, y)[0]) / 2e-6
        assert abs(fd - g[k]) <= 1e-6 + 1e-4 * abs(g[k]), (k, fd, g[k])


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 63, 64, 1000])
def test_device_gradient_matches_oracle(rrb_lib, n):
    # FP32 accumulation on the device (atomic adds in any order) against float64:
    # relative error bounded by 1e-3 of the gradient's scale.
    m = rrb_lib.MLP(0, seed=3)
    w = _params(7)
    m.set_params(w)
    np.testing.assert_array_equal(m.params(), w)
    X, y = _data(n, seed=n)
    loss, g = m.loss_grad(X, y)
    lref, gref = mlp_oracle.loss_grad(w, X, y)
    assert abs(loss - lref) <= 1e-4 * max(1.0, abs(lref))
    scale = np.abs(gref).max()
    np.testing.assert_allclose(g, gref, rtol=0, atol=1e-3 * scale)
    pred = m.predict(X)
    np.testing.assert_allclose(pred, mlp_oracle.forward(w, X)[0], rtol=1e-4, atol=1e-4)
    m.close()


@pytest.mark.gpu
def test_device_training_reduces_loss(rrb_lib):
    m = rrb_lib.MLP(0, seed=11)
    X, y = _data(20000, seed=2)
    l0, _ = m.loss_grad(X, y)
    m.train(X, y, epochs=20, batch=1024, lr=2e-3, seed=1)
    l1, _ = m.loss_grad(X, y)
    assert l1 < 0.2 * l0, (l0, l1)
    # held-out samples from the same distribution
    Xt, yt = _data(2000, seed=99)
    assert float(np.mean((m.predict(Xt) - yt) ** 2)) < 0.3 * float(np.var(yt))
    m.close()
