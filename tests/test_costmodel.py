"""Learned scheduler: MLP kernels against the NumPy oracle, training, A/B identity."""
import numpy as np
import pytest


def _random_params(rng):
    from oracle import mlp

    p = rng.normal(0, 0.3, mlp.N_PARAMS).astype(np.float32)
    p[mlp.OFF_MU:mlp.OFF_IS] = rng.normal(0, 1, mlp.NF)
    p[mlp.OFF_IS:mlp.OFF_W1] = rng.uniform(0.5, 2, mlp.NF)
    p[mlp.OFF_YMU] = 3.0
    p[mlp.OFF_YSD] = 2.0
    return p


def test_numpy_gradient_matches_finite_differences():
    from oracle import mlp

    rng = np.random.default_rng(0)
    p = _random_params(rng).astype(np.float64)
    X = rng.normal(0, 1, (40, mlp.NF))
    y = rng.normal(3, 2, 40)
    g, _ = mlp.gradient(p, X, y)
    for i in list(range(mlp.OFF_W1, mlp.OFF_W1 + 20)) + [mlp.OFF_B1 + 3, mlp.OFF_W2 + 5, mlp.OFF_B2]:
        e = np.zeros_like(p)
        e[i] = 1e-6
        num = (mlp.gradient(p + e, X, y)[1] - mlp.gradient(p - e, X, y)[1]) / 2e-6
        assert abs(num - g[i]) < 1e-5 * max(1.0, abs(num))


@pytest.mark.gpu
def test_cuda_forward_and_gradient_match_numpy():
    from cupami_b200 import costmodel
    from oracle import mlp

    rng = np.random.default_rng(1)
    p = _random_params(rng)
    X = rng.normal(0, 1, (3000, mlp.NF)).astype(np.float32)
    y = rng.normal(3, 2, 3000).astype(np.float32)
    np.testing.assert_allclose(costmodel.predict(p, X), mlp.forward(p, X), rtol=1e-4, atol=1e-4)
    g, loss = costmodel.gradient(p, X, y)
    g_ref, loss_ref = mlp.gradient(p, X, y)
    np.testing.assert_allclose(g, g_ref, rtol=2e-3, atol=2e-5)
    assert abs(loss - loss_ref) < 1e-3 * max(1.0, loss_ref)


@pytest.mark.gpu
def test_training_on_traces_beats_the_plain_key_and_keeps_output():
    import cupami_b200
    from cupami_b200 import costmodel, datasets

    train_dbs = [datasets.dense_bernoulli(n=8192, n_items=96, seed=2000 + k) for k in range(3)]
    xs, ys = zip(*(costmodel.trace(c, 0.6) for c in train_dbs))
    X, y = np.concatenate(xs), np.concatenate(ys)
    assert X.shape[0] == y.size > 500 and np.isfinite(X).all()
    params, hist = costmodel.train(X, y, epochs=300, lr=3e-3, seed=1)
    assert hist[-1] < 0.5 * hist[0]
    Xt, yt = costmodel.trace(datasets.dense_bernoulli(n=8192, n_items=96, seed=2100), 0.6)

    def spearman(a, b):
        return np.corrcoef(np.argsort(np.argsort(a)), np.argsort(np.argsort(b)))[0, 1]

    learned = spearman(costmodel.predict(params, Xt), yt)
    plain = spearman(Xt[:, 0], yt)  # feature 0 = log1p(later members), the plain order's key
    assert learned > plain
    # The order changes nothing in the output.
    csr = datasets.dense_bernoulli(n=8192, n_items=96, seed=2100)
    costmodel.use(params)
    a = cupami_b200.cuEclat(csr, 0.6)
    a.scheduler = "learned"
    a.mine()
    b = cupami_b200.cuEclat(csr, 0.6)
    b.mine()
    assert list(a.getPatterns().items()) == list(b.getPatterns().items())
    costmodel.use(None)
