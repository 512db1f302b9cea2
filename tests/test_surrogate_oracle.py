"""The FP64 surrogate oracle is pinned by central finite differences (it is
the checker of the CUDA forward/backward kernels, which have no reference
counterpart)."""
import numpy as np

from oracle import surrogate_oracle as SO


def _problem(seed=0, B=37):
    rng = np.random.default_rng(seed)
    p = rng.uniform(-0.3, 0.3, SO.NUM_PARAMS)
    X = rng.standard_normal((B, SO.IN))
    y = rng.standard_normal(B)
    return p, X, y


def test_param_count():
    assert SO.NUM_PARAMS == 128 * 10 + 128 + 128 * 128 + 128 + 2 * 128 + 2


def test_gradient_matches_finite_differences():
    p, X, y = _problem()
    L, g = SO.loss_grad(p, X, y)
    assert np.isclose(L, SO.loss(p, X, y), rtol=1e-14)
    rng = np.random.default_rng(1)
    # every bias plus a spread of weights in each layer
    idx = np.concatenate([rng.choice(1280, 40, replace=False),
                          np.arange(1280, 1408),
                          1408 + rng.choice(16384, 60, replace=False),
                          np.arange(17792, 17920),
                          17920 + np.arange(256), [18176, 18177]])
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        fd = (SO.loss(p + e, X, y) - SO.loss(p - e, X, y)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-5 * abs(g[i]), (i, fd, g[i])


def test_adam_reference_decreases_loss():
    p, X, y = _problem(2, 64)
    y = np.tanh(X[:, 0]) + 0.5 * X[:, 1]
    p2 = SO.adam_reference(p, X, y, steps=200, lr=3e-3)
    assert SO.loss(p2, X, y) < SO.loss(p, X, y) - 0.2
