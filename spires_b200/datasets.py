"""Seeded synthetic inputs with the shapes and distributions of the benchmark
workloads (no dataset files are read).

* :func:`mackey_glass` -- the Mackey-Glass delay equation
  dx/dt = 0.2 x(t-17) / (1 + x(t-17)^10) - 0.1 x(t), integrated with RK4 at
  h = 0.1 from a constant history of 1.2 plus seeded Gaussian noise (std 0.01),
  sampled every 10 sub-steps (one sample per time unit). The delayed value at
  the RK4 midpoint is the mean of the two neighbouring history samples.
* :func:`bursty_sinusoids` -- multi-channel classification sequences: every
  channel is a sum of 3 sinusoids (base frequencies U[0.01, 0.2], amplitudes
  U[0, 1], random phases) switched on and off by a two-state burst gate; each
  class shifts the base frequencies by its own offsets; sequence lengths are
  uniform integers in [len_min, len_max].
"""
from __future__ import annotations

import numpy as np


def mackey_glass(T: int, seed: int = 0, batch: int | None = None, tau: float = 17.0,
                 beta: float = 0.2, gamma: float = 0.1, n: float = 10.0, h: float = 0.1,
                 x0: float = 1.2, noise: float = 0.01, subsample: int = 10) -> np.ndarray:
    """[T] (or [batch, T]) samples of the Mackey-Glass series."""
    rng = np.random.default_rng(seed)
    B = 1 if batch is None else batch
    lag = int(round(tau / h))
    steps = T * subsample
    hist = np.empty((B, lag + steps + 1))
    hist[:, : lag + 1] = x0 + noise * rng.standard_normal((B, lag + 1))

    def f(x, xd):
        return beta * xd / (1.0 + xd ** n) - gamma * x

    for k in range(steps):
        i = lag + k
        x = hist[:, i]
        d0 = hist[:, i - lag]
        d1 = hist[:, i - lag + 1]
        dm = 0.5 * (d0 + d1)
        k1 = f(x, d0)
        k2 = f(x + 0.5 * h * k1, dm)
        k3 = f(x + 0.5 * h * k2, dm)
        k4 = f(x + h * k3, d1)
        hist[:, i + 1] = x + (h / 6.0) * (k1 + 2.0 * k2 + 2.0 * k3 + k4)
    out = hist[:, lag + subsample: lag + steps + 1: subsample][:, :T]
    return out[0] if batch is None else out


def bursty_sinusoids(num_seq: int = 500, channels: int = 13, classes: int = 10,
                     len_min: int = 20, len_max: int = 100, seed: int = 0,
                     p_switch: float = 0.1, offset_span: float = 0.015):
    """Returns (sequences: list of [len, channels] arrays, labels: [num_seq] int)."""
    rng = np.random.default_rng(seed)
    f0 = rng.uniform(0.01, 0.2, size=(channels, 3))
    offsets = rng.uniform(-offset_span, offset_span, size=(classes, channels, 3))
    labels = rng.integers(0, classes, size=num_seq)
    seqs = []
    for s in range(num_seq):
        L = int(rng.integers(len_min, len_max + 1))
        f = np.clip(f0 + offsets[labels[s]] + 0.002 * rng.standard_normal((channels, 3)),
                    0.005, 0.25)
        amp = rng.uniform(0.0, 1.0, size=(channels, 3))
        ph = rng.uniform(0.0, 2 * np.pi, size=(channels, 3))
        t = np.arange(L)[:, None, None]
        sig = (amp * np.sin(2 * np.pi * f * t + ph)).sum(axis=2)
        gate = np.empty((L, channels))
        g = rng.random(channels) < 0.5
        for k in range(L):
            flip = rng.random(channels) < p_switch
            g = np.where(flip, ~g, g)
            gate[k] = g
        seqs.append(np.ascontiguousarray(sig * gate))
    return seqs, labels


def one_step_targets(x: np.ndarray):
    """(inputs u[t] = x[t], targets y[t] = x[t+1]) from a 1-D series."""
    return x[:-1, None].copy(), x[1:, None].copy()
