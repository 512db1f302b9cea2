"""Batched hyper-parameter search on the GPU.

Two methods over the same search space and the same task:

* :func:`plain_agile` -- AGILE (Levy exploration with SPSA gradients, then
  SPSA refinement) as the reference runs it, but with many chains advanced in
  lockstep through the C ask/tell core so that every round's points are
  evaluated together in one batched simulation, each at full fidelity.
* :func:`surrogate_agile` -- the same AGILE chains, but every point they ask
  for is simulated only at the lowest fidelity; a learned surrogate (an MLP
  trained on the GPU by the library's own kernels) turns the hyper-parameters
  plus that low-fidelity loss into a predicted full-fidelity loss, which is
  what the chains are told. The asked points are pooled in waves; at the end
  of a wave the top fraction by prediction goes on to the middle fidelity,
  the top fraction of those (again by prediction, now from the middle-fidelity
  loss) to full fidelity, and every such survivor is re-simulated at full
  fidelity -- that simulation, not the surrogate, scores it and supplies the
  surrogate's next training tuples. Before the first training tuples exist
  the low-fidelity loss itself is the prediction, and `use_surrogate=False`
  keeps it so throughout (the method without the network).

An evaluation builds the candidate reservoir (seeded by the index of the point
that asked for it, so a point keeps its reservoir at every fidelity), records
its states over the training part and a validation tail of one shared
Mackey-Glass series, fits the ridge readout on the training part and scores
the one-step-ahead NRMSE on the tail; losses are log(NRMSE).
"""
from __future__ import annotations

import ctypes as C
import math
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import (CONN_RANDOM, CONN_SCALE_FREE, CONN_SMALL_WORLD, FLIF_GL, LIF_DISCRETE, AgileOpts,
               Batch, Surrogate, dptr, load, make_config)
from .datasets import mackey_glass

TOPOS = (CONN_RANDOM, CONN_SMALL_WORLD, CONN_SCALE_FREE)
DIM = 9            # encoded hyper-parameters, each in [0, 1]
FAIL_LOSS = math.log(1e3)


@dataclass
class Space:
    """The sweep's hyper-parameter space, encoded on [0, 1]^9:
    0 log N, 1 neuron model (LIF_DISCRETE below 0.5, else FLIF_GL), 2 alpha,
    3 ring length (one of `rings`), 4 spectral radius, 5 connectivity,
    6 topology (thirds), 7 log10 ridge lambda, 8 log10 input gain (the
    reference's own AGILE space also searches the gain and lambda)."""
    n_range: tuple = (500, 8000)
    rings: tuple = (128, 256, 512, 1024)
    alpha: tuple = (0.3, 1.0)
    rho: tuple = (0.5, 1.5)
    conn: tuple = (0.02, 0.2)
    log10_lambda: tuple = (-8.0, 0.0)
    log10_gain: tuple = (-2.5, 0.0)

    def decode(self, th):
        th = np.clip(np.asarray(th, np.float64), 0.0, 1.0)
        lo, hi = math.log(self.n_range[0]), math.log(self.n_range[1])
        return {
            "n": int(round(math.exp(lo + th[0] * (hi - lo)))),
            "neuron": FLIF_GL if th[1] >= 0.5 else LIF_DISCRETE,
            "alpha": self.alpha[0] + th[2] * (self.alpha[1] - self.alpha[0]),
            "L": self.rings[min(len(self.rings) - 1, int(th[3] * len(self.rings)))],
            "rho": self.rho[0] + th[4] * (self.rho[1] - self.rho[0]),
            "conn": self.conn[0] + th[5] * (self.conn[1] - self.conn[0]),
            "topo": TOPOS[min(2, int(th[6] * 3))],
            "lam": 10.0 ** (self.log10_lambda[0] + th[7] * (self.log10_lambda[1] -
                                                          self.log10_lambda[0])),
            "gain": 10.0 ** (self.log10_gain[0] + th[8] * (self.log10_gain[1] -
                                                         self.log10_gain[0])),
        }

    def config(self, th):
        d = self.decode(th)
        if d["neuron"] == FLIF_GL:
            p = (1.0, 0.0, 0.0, 20.0, d["alpha"], float(d["L"]), 0.1, 2.0)
        else:
            p = (0.0, 1.0, 0.9, 0.0)
        return make_config(d["n"], 1, 1, rho=d["rho"], ei=0.5, gamma=d["gain"], conn=d["conn"],
                           dt=1.0, topo=d["topo"], neuron=d["neuron"], nparams=p), d

    def features(self, th):
        """Hyper-parameter part of the surrogate input (9 values in [0, 1])."""
        th = np.clip(np.atleast_2d(np.asarray(th, np.float64)), 0.0, 1.0)
        f = th.copy()
        f[:, 1] = (th[:, 1] >= 0.5).astype(np.float64)
        f[:, 3] = np.minimum(len(self.rings) - 1, np.floor(th[:, 3] * len(self.rings))) / \
            max(1, len(self.rings) - 1)
        f[:, 6] = np.minimum(2, np.floor(th[:, 6] * 3)) / 2.0
        return f


@dataclass
class Task:
    """One-step-ahead prediction of one shared Mackey-Glass series."""
    length: int = 16000
    val: int = 1000
    washout: int = 200
    seed: int = 7
    x: np.ndarray = field(default=None, repr=False)

    def __post_init__(self):
        if self.x is None:
            self.x = mackey_glass(self.length + self.val + 1, seed=self.seed)

    def series(self, T):
        """(u, y) of T training steps followed by the validation tail."""
        x = self.x[: T + self.val + 1]
        return np.ascontiguousarray(x[:-1, None]), np.ascontiguousarray(x[1:, None])


@dataclass
class EvalStats:
    evals: int = 0
    neuron_steps: float = 0.0
    sim_s: float = 0.0     # whole evaluate() calls
    build_s: float = 0.0   # reservoir construction (host topology + device upload)
    build_wait_s: float = 0.0  # part of it the evaluation waited for (not overlapped)
    construct_s: float = 0.0  # ... of which host construction (all host threads)
    setup_s: float = 0.0      # ... of which device layouts and uploads
    fit_s: float = 0.0     # batched simulation + ridge fits + readouts
    calls: int = 0


class Evaluator:
    """Scores candidates in batches (chunked so that the recorded states of
    one batch stay within `state_bytes` of device memory)."""

    def __init__(self, space: Space, task: Task, seed: int = 1, state_bytes: float = 24e9):
        self.space = space
        self.task = task
        self.seed = seed
        self.state_bytes = state_bytes
        self.stats = EvalStats()

    def instance_seed(self, cid):
        return int((self.seed * 0x9E3779B1 + int(cid) * 0x85EBCA77) & 0x7FFFFFFF) or 1

    def evaluate(self, thetas, T, ids):
        return self.evaluate_rungs(thetas, (T,), ids)[0]

    def evaluate_rungs(self, thetas, rungs, ids):
        """Losses of the same candidates at several training lengths, each
        reservoir built once (list of arrays, one per length)."""
        thetas = np.atleast_2d(thetas)
        outs = [np.full(len(thetas), FAIL_LOSS) for _ in rungs]
        if len(thetas) == 0:
            return outs
        total = max(rungs) + self.task.val
        cfgs, decs = zip(*[self.space.config(th) for th in thetas])
        chunks, cur, acc = [], [], 0.0
        for k in range(len(thetas)):
            b = total * (((decs[k]["n"] + 31) // 32) * 32) * 8.0
            if cur and acc + b > self.state_bytes:
                chunks.append(cur)
                cur, acc = [], 0.0
            cur.append(k)
            acc += b
        if cur:
            chunks.append(cur)
        t0 = time.perf_counter()

        def build(ch):
            tb = time.perf_counter()
            b = Batch([cfgs[k] for k in ch], [self.instance_seed(ids[k]) for k in ch])
            return b, tb, time.perf_counter()

        # the next chunk's reservoirs are built (host construction on all
        # cores, device set-up) while the current chunk simulates and fits
        pool = ThreadPoolExecutor(max_workers=1)
        nxt = pool.submit(build, chunks[0])
        for ci, ch in enumerate(chunks):
            tq = time.perf_counter()
            batch, tb, tf = nxt.result()
            tw = time.perf_counter()
            self.stats.build_wait_s += tw - tq  # construction not hidden
            if ci + 1 < len(chunks):
                nxt = pool.submit(build, chunks[ci + 1])
            c_ms, s_ms = batch.timing()
            self.stats.construct_s += c_ms / 1e3
            self.stats.setup_s += s_ms / 1e3
            lams = [decs[k]["lam"] for k in ch]
            for out, T in zip(outs, rungs):
                u, y = self.task.series(T)
                yv = y[T:, 0]
                sd = yv.std()
                Y, _ = batch.fit_predict([u] * len(ch), [y] * len(ch), [T] * len(ch), lams,
                                         washout=min(self.task.washout, T // 2))
                for j, k in enumerate(ch):
                    e = Y[j][T:, 0] - yv
                    nr = math.sqrt(float(np.mean(e * e))) / (sd if sd > 0 else 1.0)
                    out[k] = (min(math.log(nr), FAIL_LOSS) if np.isfinite(nr) and nr > 0
                              else FAIL_LOSS)
                self.stats.neuron_steps += sum(decs[k]["n"] for k in ch) * float(
                    T + self.task.val)
            batch.close()
            self.stats.build_s += tf - tb
            self.stats.fit_s += time.perf_counter() - tw
        pool.shutdown()
        self.stats.sim_s += time.perf_counter() - t0
        self.stats.evals += len(thetas) * len(rungs)
        self.stats.calls += 1
        return outs


@dataclass
class SearchResult:
    best_loss: float
    best_theta: np.ndarray
    wall_s: float
    evals: int
    history: list        # (elapsed s, best full-fidelity loss so far)
    extra: dict = field(default_factory=dict)

    @property
    def best_nrmse(self):
        return math.exp(self.best_loss)

    def time_to(self, loss):
        """First elapsed time at which the best loss was <= loss (None if never)."""
        for t, b in self.history:
            if b <= loss:
                return t
        return None


def default_opts():
    # steps on the unit cube: Levy lengths in [0.01, 0.5], SPSA probes of 0.02
    return AgileOpts(1.3, 1e-2, 0.5, 10.0, 0.9, 2e-2, 20, 5, 2e-2, 1, 0, 0)


def _agile_start(chains, seed, opts):
    rng = np.random.default_rng(seed)
    th0 = np.ascontiguousarray(rng.uniform(0.0, 1.0, (chains, DIM)))
    opts = opts or default_opts()
    seeds = (C.c_uint64 * chains)(*[int(s) for s in rng.integers(1, 2**62, chains)])
    lib = load()
    h = C.c_void_p()
    st = lib.spires_ext_agile_batch_create(chains, DIM, dptr(th0), dptr(np.zeros(DIM)),
                                           dptr(np.ones(DIM)), C.byref(opts), seeds, C.byref(h))
    if st != 0:
        raise RuntimeError(f"spires_ext_agile_batch_create failed: {st}")
    return lib, h


def plain_agile(ev: Evaluator, chains: int = 16, T: int = 16000, seed: int = 0,
                opts: AgileOpts | None = None, max_points: int | None = None) -> SearchResult:
    """Lockstep AGILE chains, every evaluation at full fidelity T."""
    lib, h = _agile_start(chains, seed, opts)
    pts = np.empty((2 * chains, DIM))
    owner = (C.c_int * (2 * chains))()
    best, best_th, hist, evals = math.inf, None, [], 0
    t0 = time.perf_counter()
    try:
        while max_points is None or evals < max_points:
            n = lib.spires_ext_agile_batch_ask(h, dptr(pts), owner)
            if n <= 0:
                break
            losses = ev.evaluate(pts[:n], T, np.arange(evals, evals + n))
            evals += n
            k = int(np.argmin(losses))
            if losses[k] < best:
                best, best_th = float(losses[k]), pts[k].copy()
            hist.append((time.perf_counter() - t0, best))
            lib.spires_ext_agile_batch_tell(h, dptr(np.ascontiguousarray(losses)))
    finally:
        lib.spires_ext_agile_batch_destroy(h)
    return SearchResult(best, best_th, time.perf_counter() - t0, evals, hist, {"points": evals})


def surrogate_agile(ev: Evaluator, chains: int = 16, rungs=(1000, 4000, 16000), keep: float = 0.1,
                    max_points: int = 4096, waves: int = 8, seed: int = 0,
                    opts: AgileOpts | None = None, use_surrogate: bool = True, epochs: int = 200,
                    calibration: int = 8, kappa: float = 1.0,
                    prescreen: float = 0.0, tell_optimistic: bool = False) -> SearchResult:
    """Surrogate-guided multi-fidelity AGILE (see module doc). The chains start
    from the same points with the same seeds as :func:`plain_agile`.

    Cut r (after rung r) ranks by its own network, an MLP 10 -> 128 -> 128 -> 2
    mapping the 9 hyper-parameter features plus the rung-r loss to the mean
    and log-variance of the full-fidelity loss. So that the training tuples
    are not only the best points, the chains' start points all go through
    every rung (their full-fidelity losses are what the chains are told for
    them; the networks train on them before the first wave), and every wave
    carries `calibration` further seeded random points through every rung.
    Cuts rank by the optimistic score mean - kappa * std, so that points the
    network is unsure about still get simulated.

    prescreen > 0 adds a cut before any simulation: once the networks have
    trained, a further network maps the 9 hyper-parameter features alone to
    the full-fidelity loss, and of each round's asked points only the best
    fraction `prescreen` by its optimistic score (plus `calibration` random
    ones) is built and simulated at the lowest fidelity; the chains are told
    that network's prediction for the others, which are neither built nor
    pooled.

    tell_optimistic tells the chains the optimistic score mean - kappa * std
    instead of the predicted mean, so that regions the network is unsure
    about attract them."""
    lib, h = _agile_start(chains, seed, opts)
    ncut = len(rungs) - 1
    nets = [Surrogate(seed=seed + r) for r in range(ncut)] if use_surrogate else None
    pre_net = Surrogate(seed=seed + 97) if (use_surrogate and prescreen > 0.0) else None
    X_pre = []
    screened = 0
    trained = False
    rng = np.random.default_rng(seed + 7)
    pts = np.empty((2 * chains, DIM))
    owner = (C.c_int * (2 * chains))()
    X_tr = [[] for _ in range(ncut)]
    y_tr = []
    pool_th, pool_l0, pool_id = [], [], []
    best, best_th, hist, evals, asked = math.inf, None, [], 0, 0
    pred_rmse, low_rmse = [], []
    wave_size = max(1, max_points // max(1, waves))
    wave_asked = 0
    t0 = time.perf_counter()

    def net_input(th, low):
        return np.concatenate([ev.space.features(th), np.asarray(low, np.float64)[:, None]],
                              axis=1).astype(np.float32)

    def predict(r, th, low, optimistic=False):
        if not trained:
            return np.asarray(low, np.float64)
        m, v = nets[r].predict(net_input(th, low), bf16=True)
        m = m.astype(np.float64)
        if optimistic:
            m = m - kappa * np.exp(0.5 * np.clip(v.astype(np.float64), -20.0, 20.0))
        return m

    def cut_wave(th, l0, pid):
        # pid: asked index of every point, the seed of its reservoir at every rung
        nonlocal best, best_th, evals, trained
        n = len(th)
        lows = [l0]
        sel = np.arange(n)
        cal = (rng.choice(n, size=min(calibration, n), replace=False)
               if nets is not None else np.array([], dtype=np.int64))
        for r in range(ncut):
            est = predict(r, th[sel], lows[r][sel], optimistic=True)
            nk = max(1, int(math.ceil(keep * len(sel))))
            sel = np.union1d(sel[np.argsort(est, kind="stable")[:nk]], cal)
            l = np.full(n, np.nan)
            l[sel] = ev.evaluate(th[sel], rungs[r + 1], pid[sel])
            evals += len(sel)
            lows.append(l)
        full = lows[-1][sel]
        k = int(np.argmin(full))
        if full[k] < best:
            best, best_th = float(full[k]), th[sel[k]].copy()
        hist.append((time.perf_counter() - t0, best))
        if nets is None:
            return
        new_X = [net_input(th[sel], lows[r][sel]) for r in range(ncut)]
        if trained:
            # error on tuples the network has not trained on yet, next to the
            # error of taking the rung-0 loss itself as the prediction
            m, _ = nets[0].predict(new_X[0], bf16=True)
            pred_rmse.append(float(np.sqrt(np.mean((m - full) ** 2))))
            low_rmse.append(float(np.sqrt(np.mean((lows[0][sel] - full) ** 2))))
        y_tr.extend(full.tolist())
        ya = np.asarray(y_tr, np.float32)
        for r in range(ncut):
            X_tr[r].extend(list(new_X[r]))
            nets[r].train(np.asarray(X_tr[r], np.float32), ya, epochs=epochs,
                          batch=min(256, len(ya)), lr=1e-3, seed=seed + 31 * len(hist) + r)
        if pre_net is not None:
            X_pre.extend(list(net_input(th[sel], np.zeros(len(sel)))))
            pre_net.train(np.asarray(X_pre, np.float32), ya, epochs=epochs,
                          batch=min(256, len(ya)), lr=1e-3, seed=seed + 31 * len(hist) + 17)
        trained = True

    try:
        # the chains' start points: every rung, told their full-fidelity loss
        n = lib.spires_ext_agile_batch_ask(h, dptr(pts), owner)
        if n > 0:
            th = pts[:n].copy()
            lows = ev.evaluate_rungs(th, rungs, np.arange(n))
            evals += n * len(rungs)
            asked += n
            full = lows[-1]
            k = int(np.argmin(full))
            best, best_th = float(full[k]), th[k].copy()
            hist.append((time.perf_counter() - t0, best))
            if nets is not None:
                y_tr.extend(full.tolist())
                for r in range(ncut):
                    X_tr[r].extend(list(net_input(th, lows[r])))
                    nets[r].train(np.asarray(X_tr[r], np.float32), np.asarray(y_tr, np.float32),
                                  epochs=epochs, batch=min(256, len(y_tr)), lr=1e-3,
                                  seed=seed + r)
                if pre_net is not None:
                    X_pre.extend(list(net_input(th, np.zeros(n))))
                    pre_net.train(np.asarray(X_pre, np.float32), np.asarray(y_tr, np.float32),
                                  epochs=epochs, batch=min(256, len(y_tr)), lr=1e-3,
                                  seed=seed + 97)
                trained = True
            lib.spires_ext_agile_batch_tell(h, dptr(np.ascontiguousarray(full)))
        while asked < max_points:
            n = lib.spires_ext_agile_batch_ask(h, dptr(pts), owner)
            if n <= 0:
                break
            th = pts[:n].copy()
            ids = np.arange(asked, asked + n)
            asked += n
            est = np.empty(n)
            run = np.arange(n)
            if pre_net is not None and trained:
                m, v = pre_net.predict(net_input(th, np.zeros(n)), bf16=True)
                score = m.astype(np.float64) - kappa * np.exp(
                    0.5 * np.clip(v.astype(np.float64), -20.0, 20.0))
                nk = max(1, int(math.ceil(prescreen * n)))
                cal = rng.choice(n, size=min(calibration, n), replace=False)
                run = np.union1d(np.argsort(score, kind="stable")[:nk], cal)
                rest = np.setdiff1d(np.arange(n), run)
                est[rest] = (score if tell_optimistic else m.astype(np.float64))[rest]
                screened += len(rest)
            l0 = ev.evaluate(th[run], rungs[0], ids[run])
            evals += len(run)
            est[run] = predict(0, th[run], l0, optimistic=tell_optimistic)
            lib.spires_ext_agile_batch_tell(h, dptr(np.ascontiguousarray(est)))
            pool_th.append(th[run])
            pool_l0.append(l0)
            pool_id.append(ids[run])
            wave_asked += n  # waves are counted in asked points, pooled or screened
            if wave_asked >= wave_size:
                cut_wave(np.concatenate(pool_th), np.concatenate(pool_l0),
                         np.concatenate(pool_id))
                pool_th, pool_l0, pool_id = [], [], []
                wave_asked = 0
        if pool_th:
            cut_wave(np.concatenate(pool_th), np.concatenate(pool_l0), np.concatenate(pool_id))
    finally:
        lib.spires_ext_agile_batch_destroy(h)
        if nets is not None:
            for net in nets:
                net.close()
        if pre_net is not None:
            pre_net.close()
    extra = {"surrogate_rmse": pred_rmse, "low_fidelity_rmse": low_rmse, "tuples": len(y_tr),
             "points": asked, "screened_out": screened}
    return SearchResult(best, best_th, time.perf_counter() - t0, evals, hist, extra)
