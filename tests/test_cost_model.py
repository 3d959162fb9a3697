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


# ---- features, autotuner table and the trained model --------------------------------

def test_page_features_are_consistent(rrb_lib):
    s = rrb_lib.Scene(2, 3, n_pages=2, page_scale=0.1, paths_scale=0.01)
    for pg in range(2):
        rows = [rrb_lib.page_features(s.view, pg, t) for t in rrb_lib.TILE_SHAPES]
        for k, f in enumerate(rows):
            assert f[21:24].tolist() == [float(j == k) for j in range(3)]
            assert abs(f[13:21].sum() - 1.0) < 1e-5 and abs(f[12] - (1.0 - f[13])) < 1e-5
            n = int(np.sum(s.path_page == pg))
            assert abs(f[1] - np.log1p(n)) < 1e-4
            w, h = int(s.page_width[pg]), int(s.page_height[pg])
            assert abs(f[0] - np.log1p(w * h)) < 1e-3
        # Only the tile-dependent features differ between shapes.
        assert np.array_equal(rows[0][:12], rows[1][:12]) and np.array_equal(rows[0][:12], rows[2][:12])


def test_autotuner_table_picks_the_fastest_shape_per_bin():
    from rrb.autotune import bins, build_table

    rng = np.random.default_rng(0)
    X = np.zeros((300, 3, 24), np.float32)
    X[:, :, 0] = rng.uniform(12, 18, 300)[:, None]
    X[:, :, 5] = X[:, :, 0] + rng.uniform(-8, 0, 300)[:, None]
    T = rng.uniform(1, 2, (300, 3))
    T[:, 1] *= 0.5  # 32x32 fastest everywhere
    table = build_table(X, T)
    keys = np.unique(bins(X[:, 0]))
    assert all(table[k] == 1 for k in keys)
    assert all(table[k] == 2 for k in set(range(16)) - set(keys.tolist()))  # empty bins: 64x16


def test_cost_model_round_trips(tmp_path):
    from rrb.autotune import CostModel

    m = CostModel(np.arange(5825, dtype=np.float32), np.ones(24, np.float32), np.full(24, 2, np.float32), 0.5, 1.5,
                  np.arange(16, dtype=np.int32) % 3)
    m.save(tmp_path / "m.npz")
    r = CostModel.load(tmp_path / "m.npz")
    assert np.array_equal(r.params, m.params) and r.y_mean == 0.5 and r.y_std == 1.5
    assert np.array_equal(r.table, m.table)


def test_host_forward_matches_oracle(rrb_lib):
    w = _params(13)
    X, _ = _data(300, seed=4)
    got = rrb_lib.MLP.predict_host(w, X)
    np.testing.assert_allclose(got, mlp_oracle.forward(w, X)[0], rtol=1e-4, atol=1e-4)


@pytest.mark.gpu
def test_host_forward_equals_device_forward(rrb_lib):
    w = _params(17)
    X, _ = _data(777, seed=8)
    m = rrb_lib.MLP(0)
    m.set_params(w)
    dev = m.predict(X)
    m.close()
    assert np.array_equal(dev.view(np.uint32), rrb_lib.MLP.predict_host(w, X).view(np.uint32))


@pytest.mark.gpu
def test_trained_model_beats_the_default_tile_on_held_out_pages(rrb_lib):
    """The committed model (trained on 50,100 (page, tile) pairs) against the
    5,000 held-out pages of the sweep: its per-page tile choice costs less
    measured device time than the fixed 64x16 default (the method without a
    tuner), and its time predictions stay within 20% on average. It does NOT
    beat the autotuner table on tile choice: the table is within 0.7% of the
    best shape per page, and the model's choices cost 0.2% more than the
    table's (model_vs_table 0.998); this pins that it stays within 2% of it."""
    from pathlib import Path

    from rrb.autotune import CostModel, evaluate

    root = Path(__file__).resolve().parents[1]
    model = CostModel.load(root / "pdf-raster_b200" / "rrb" / "cost_model.npz")
    d = np.load(root / "tests" / "golden" / "cost_model_holdout.npz")
    rep = evaluate(model, d["X"], d["ms"])
    assert rep["pages"] == 5000
    assert rep["model_vs_default"] > 1.05
    assert 0.98 < rep["model_vs_table"] < 1.0 + 1e-3  # as good as the table, not better
    assert rep["mape"] < 0.2
    # The device and host forward passes give the same choices.
    X = d["X"][:200]
    host = rrb_lib.MLP.predict_host(model.params, model.norm(X.reshape(-1, 24))).reshape(-1, 3)
    assert np.array_equal(np.argmin(host, 1), model.choose(X))
