"""CPU oracle of the search surrogate (test infrastructure only).

FP64 numpy restatement of the MLP 10 -> 128 -> 128 -> 2 with exact (erf)
GELU and the Gaussian negative log-likelihood
    loss = mean_s 0.5 * (v_s + (y_s - m_s)^2 * exp(-v_s)),
with the parameter layout of spires_ext_mlp (W1[128][10], b1[128],
W2[128][128], b2[128], W3[2][128], b3[2], concatenated). The network has no
counterpart in the reference; this oracle is pinned by central finite
differences instead (tests/test_surrogate_oracle.py) and is the checker of the
CUDA forward and backward kernels. Nothing in the library imports it.
"""
from __future__ import annotations

import math

import numpy as np

IN, HID, OUT = 10, 128, 2
SHAPES = [("W1", (HID, IN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)),
          ("W3", (OUT, HID)), ("b3", (OUT,))]
NUM_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)

_erf = np.vectorize(math.erf, otypes=[np.float64])


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    out, o = {}, 0
    for name, shape in SHAPES:
        k = int(np.prod(shape))
        out[name] = p[o:o + k].reshape(shape)
        o += k
    return out


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    cdf = 0.5 * (1.0 + _erf(x / math.sqrt(2.0)))
    pdf = np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)
    return cdf + x * pdf


def forward(p, X):
    P = unpack(p)
    X = np.asarray(X, dtype=np.float64)
    z1 = X @ P["W1"].T + P["b1"]
    h1 = gelu(z1)
    z2 = h1 @ P["W2"].T + P["b2"]
    h2 = gelu(z2)
    o = h2 @ P["W3"].T + P["b3"]
    return o, (X, z1, h1, z2, h2)


def loss(p, X, y):
    o, _ = forward(p, X)
    m, v = o[:, 0], o[:, 1]
    r = np.asarray(y, np.float64) - m
    return float(np.mean(0.5 * (v + r * r * np.exp(-v))))


def loss_grad(p, X, y):
    P = unpack(p)
    o, (X, z1, h1, z2, h2) = forward(p, X)
    B = X.shape[0]
    m, v = o[:, 0], o[:, 1]
    r = np.asarray(y, np.float64) - m
    iv = np.exp(-v)
    L = float(np.mean(0.5 * (v + r * r * iv)))
    do = np.stack([-r * iv, 0.5 * (1.0 - r * r * iv)], axis=1) / B
    gW3 = do.T @ h2
    gb3 = do.sum(axis=0)
    dz2 = (do @ P["W3"]) * gelu_grad(z2)
    gW2 = dz2.T @ h1
    gb2 = dz2.sum(axis=0)
    dz1 = (dz2 @ P["W2"]) * gelu_grad(z1)
    gW1 = dz1.T @ X
    gb1 = dz1.sum(axis=0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return L, g


def adam_reference(p, X, y, steps, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """Full-batch Adam in FP64 (for trajectory checks on tiny problems)."""
    p = np.array(p, dtype=np.float64)
    m1 = np.zeros_like(p)
    m2 = np.zeros_like(p)
    for t in range(1, steps + 1):
        _, g = loss_grad(p, X, y)
        m1 = b1 * m1 + (1 - b1) * g
        m2 = b2 * m2 + (1 - b2) * g * g
        p -= lr * (m1 / (1 - b1 ** t)) / (np.sqrt(m2 / (1 - b2 ** t)) + eps)
    return p
