"""Selector MLP kernels against the FP64 CPU oracle (forward, loss gradient)
and a training run that must fit a known target."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def selector(sg):
    from sygraph_b200 import selector
    return selector


def _data(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, 12)).astype(np.float32)
    T = rng.normal(size=(n, 6)).astype(np.float32)
    M = (rng.random((n, 6)) > 0.2).astype(np.float32)
    return X, T, M


def test_param_layout(selector):
    from oracle import mlp as omlp
    assert selector.PARAM_COUNT == sum(int(np.prod(s)) for _, s in omlp.SHAPES)
    assert selector.TRAINABLE_COUNT == selector.PARAM_COUNT - 48


def test_forward_matches_fp64_oracle(selector):
    from oracle import mlp as omlp
    m = selector.Mlp()
    X, _, _ = _data(300, 1)
    m.set_normalisation(X)
    y = m.forward(X)
    y64, _ = omlp.forward(m.params.astype(np.float64), X)
    np.testing.assert_allclose(y, y64, rtol=1e-4, atol=1e-4)


def test_gradient_matches_fp64_oracle(selector):
    from oracle import mlp as omlp
    m = selector.Mlp()
    X, T, M = _data(257, 2)
    m.set_normalisation(X)
    loss, g = m.gradient(X, T, M)
    loss64, g64 = omlp.loss_and_grad(m.params.astype(np.float64), X, T, M)
    assert abs(loss - loss64) <= 1e-4 * max(1.0, abs(loss64))
    t = selector.TRAINABLE_COUNT
    np.testing.assert_allclose(g[:t], g64[:t], rtol=2e-3, atol=2e-6)
    assert np.all(g[t:] == 0)


def test_training_fits_a_smooth_target(selector):
    rng = np.random.default_rng(3)
    X = rng.uniform(-1, 1, size=(2000, 12)).astype(np.float32)
    W = rng.normal(size=(12, 6)).astype(np.float32)
    T = np.tanh(X @ W).astype(np.float32)
    M = np.ones_like(T)
    m = selector.Mlp()
    m.set_normalisation(X)
    loss0, _ = m.gradient(X, T, M)
    loss = m.train(X, T, M, steps=1500, lr=3e-3)
    assert loss < 0.1 * loss0
    # argmin agreement with the target on held-out points
    Xt = rng.uniform(-1, 1, size=(500, 12)).astype(np.float32)
    agree = (m.choose(Xt) == np.tanh(Xt @ W).argmin(1)).mean()
    assert agree > 0.7
