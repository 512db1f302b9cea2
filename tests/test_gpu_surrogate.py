"""The surrogate network's CUDA kernels against the FP64 CPU oracle: forward
outputs, the NLL and its gradient, Adam trajectories, and the BF16 inference
path. All calls go through the C ABI of libspires.so."""
import numpy as np
import pytest

import spires_b200 as sp
from oracle import surrogate_oracle as SO

pytestmark = pytest.mark.gpu


def data(B, seed=0):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((B, 10)).astype(np.float32)
    y = (np.tanh(X[:, 0]) + 0.3 * X[:, 1] * X[:, 2] + 0.1 * rng.standard_normal(B)).astype(
        np.float32)
    return X, y


def test_param_layout_and_init():
    s = sp.Surrogate(seed=3)
    assert s.num_params == SO.NUM_PARAMS
    p = s.params()
    P = SO.unpack(p)
    assert np.all(np.abs(P["W1"]) <= 1 / np.sqrt(10) + 1e-7)
    assert np.all(np.abs(P["W2"]) <= 1 / np.sqrt(128) + 1e-7)
    assert np.std(P["W2"]) > 0.03
    assert np.array_equal(sp.Surrogate(seed=3).params(), p)  # seeded
    assert not np.array_equal(sp.Surrogate(seed=4).params(), p)


@pytest.mark.parametrize("B", [1, 37, 300, 1000])
def test_loss_and_gradient_match_oracle(B):
    s = sp.Surrogate(seed=1)
    p = s.params()
    X, y = data(B, seed=B)
    L, g = s.loss_grad(X, y)
    Lo, go = SO.loss_grad(p.astype(np.float64), X.astype(np.float64), y.astype(np.float64))
    # FP32 kernels against FP64: relative 1e-5 on the loss, 1e-4 of the
    # gradient's scale on every component
    assert abs(L - Lo) <= 1e-5 * max(1.0, abs(Lo))
    scale = np.abs(go).max()
    assert np.max(np.abs(g - go)) <= 1e-4 * scale, np.max(np.abs(g - go)) / scale
    assert np.linalg.norm(g - go) <= 1e-4 * np.linalg.norm(go)


def test_forward_fp32_and_bf16_match_oracle():
    s = sp.Surrogate(seed=2)
    p = s.params()
    X, _ = data(513, seed=5)
    o, _ = SO.forward(p.astype(np.float64), X.astype(np.float64))
    m32, v32 = s.predict(X, bf16=False)
    assert np.max(np.abs(m32 - o[:, 0])) <= 1e-5 * max(1.0, np.abs(o[:, 0]).max())
    assert np.max(np.abs(v32 - o[:, 1])) <= 1e-5 * max(1.0, np.abs(o[:, 1]).max())
    m16, v16 = s.predict(X, bf16=True)
    # BF16 operands (8-bit mantissa), FP32 sums: a few parts in a thousand
    assert np.max(np.abs(m16 - o[:, 0])) <= 2e-2 * max(1.0, np.abs(o[:, 0]).max())
    assert np.max(np.abs(v16 - o[:, 1])) <= 2e-2 * max(1.0, np.abs(o[:, 1]).max())
    assert not np.array_equal(m16, m32)


def test_adam_trajectory_matches_oracle():
    s = sp.Surrogate(seed=7)
    p0 = s.params()
    X, y = data(64, seed=9)
    # one minibatch per epoch = full-batch Adam, as the oracle runs it
    s.train(X, y, epochs=5, batch=64, lr=1e-3, seed=0)
    p5 = s.params()
    po = SO.adam_reference(p0.astype(np.float64), X.astype(np.float64), y.astype(np.float64), 5,
                           lr=1e-3)
    # five steps of at most ~lr each: agreement to well below one step; a
    # component whose gradient is within FP32 rounding of zero may take an
    # Adam step of the other sign, so the bound on every component is 5 lr
    d = np.abs(p5 - po)
    assert np.quantile(d, 0.999) <= 1e-5
    assert d.max() <= 5.5e-3
    assert np.max(np.abs(p5 - p0)) > 1e-4


def test_training_fits_a_noisy_function():
    X, y = data(4096, seed=11)
    Xv, yv = data(1024, seed=12)
    s = sp.Surrogate(seed=0)
    before = float(np.mean((s.predict(Xv, bf16=False)[0] - yv) ** 2))
    s.train(X, y, epochs=60, batch=256, lr=1e-3, seed=1)
    m, v = s.predict(Xv, bf16=True)
    after = float(np.mean((m - yv) ** 2))
    assert after < 0.25 * before
    assert after < 0.05
    # the variance head learns the noise level (std 0.1 -> logvar ~ -4.6)
    assert -6.5 < float(np.median(v)) < -2.5
    assert s.lib.spires_ext_mlp_kernel_launches(s.h) > 0
