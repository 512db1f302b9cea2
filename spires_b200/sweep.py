"""Hyper-parameter sweep workloads over many reservoirs.

:func:`sweep_space` draws a seeded population of uneven reservoirs (size
log-uniform, LIF_DISCRETE or FLIF_GL, fractional order, ring length, spectral
radius, connectivity, topology) each with its own Mackey-Glass series and
one-step-ahead targets; :func:`run_sweep` builds them as one batch, fits every
ridge readout from one batched simulation and scores every instance by NRMSE on
a held-out tail of its series.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import CONN_RANDOM, CONN_SCALE_FREE, CONN_SMALL_WORLD, FLIF_GL, LIF_DISCRETE
from . import Batch, make_config
from .datasets import mackey_glass

GL_BASE = (1.0, 0.0, 0.0, 20.0, 0.7, 512.0, 0.1, 2.0)  # [V_th, V_reset, V_rest, tau_m, alpha, T_mem, bias, t_ref]
LIF_BASE = (0.0, 1.0, 0.9, 0.0)                        # [V_0, V_th, leak_rate, bias]
TOPOLOGIES = (CONN_RANDOM, CONN_SMALL_WORLD, CONN_SCALE_FREE)


@dataclass
class Instance:
    n: int
    neuron: int
    alpha: float
    L: int
    rho: float
    conn: float
    topo: int
    T: int
    seed: int
    mg_seed: int
    cfg: object = field(default=None, repr=False)


def instance_config(n, neuron, alpha, L, rho, conn, topo, gamma=0.5, ei=0.5):
    if neuron == FLIF_GL:
        p = list(GL_BASE)
        p[4] = alpha
        p[5] = float(L)
    else:
        p = list(LIF_BASE)
    return make_config(n, 1, 1, rho=rho, ei=ei, gamma=gamma, conn=conn, dt=1.0, topo=topo,
                       neuron=neuron, nparams=p)


def sweep_space(count: int = 256, seed: int = 2024, n_range=(500, 8000), t_range=(2000, 10000),
                rings=(128, 256, 512, 1024), conn_range=(0.02, 0.2)) -> list[Instance]:
    """Seeded population of `count` sweep instances."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(round(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1])))))
        neuron = (LIF_DISCRETE, FLIF_GL)[int(rng.integers(0, 2))]
        inst = Instance(n=n, neuron=neuron, alpha=float(rng.uniform(0.3, 1.0)),
                        L=int(rng.choice(rings)), rho=float(rng.uniform(0.5, 1.5)),
                        conn=float(rng.uniform(*conn_range)),
                        topo=TOPOLOGIES[int(rng.integers(0, 3))],
                        T=int(rng.integers(t_range[0], t_range[1] + 1)),
                        seed=int(rng.integers(1, 2**31 - 1)),
                        mg_seed=int(rng.integers(0, 2**31 - 1)))
        inst.cfg = instance_config(inst.n, inst.neuron, inst.alpha, inst.L, inst.rho, inst.conn,
                                   inst.topo)
        out.append(inst)
    return out


def series_for(insts: list[Instance], seed: int = 7):
    """Mackey-Glass series of every instance (one batched integration, each
    instance its own noisy history), as (u, y) one-step-ahead pairs."""
    Tmax = max(i.T for i in insts) + 1
    X = mackey_glass(Tmax, seed=seed, batch=len(insts))
    us, ys = [], []
    for k, inst in enumerate(insts):
        x = X[k, : inst.T + 1]
        us.append(np.ascontiguousarray(x[:-1, None]))
        ys.append(np.ascontiguousarray(x[1:, None]))
    return us, ys


def nrmse(y, yhat):
    y = np.asarray(y).ravel()
    yhat = np.asarray(yhat).ravel()
    sd = y.std()
    return float(np.sqrt(np.mean((y - yhat) ** 2)) / (sd if sd > 0 else 1.0))


def run_sweep(insts: list[Instance], washout: int = 500, val_frac: float = 0.2,
              lam: float = 1e-6, batch: Batch | None = None):
    """Fit and score every instance; returns a dict with timings and scores.

    Each series is split into a training head and a validation tail; one
    batched simulation records the states of the whole series, the ridge is
    fitted on the head (states after `washout`) and the readout of the tail
    is scored."""
    t0 = time.perf_counter()
    b = batch or Batch([i.cfg for i in insts], [i.seed for i in insts])
    t_build = time.perf_counter() - t0
    us, ys = series_for(insts)
    heads = [int(i.T * (1.0 - val_frac)) for i in insts]
    t1 = time.perf_counter()
    # one recorded simulation per instance serves the fit (head) and the score
    Y, _ = b.fit_predict(us, ys, heads, lam, washout=washout)
    t2 = time.perf_counter()
    scores = [nrmse(y[h:], Yk[h:, :1]) for y, Yk, h in zip(ys, Y, heads)]
    return {"batch": b, "build_s": t_build, "fit_score_s": t2 - t1,
            "nrmse": np.asarray(scores), "heads": heads}
