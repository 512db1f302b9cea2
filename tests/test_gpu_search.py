"""Batched search on the GPU (small scale): the evaluator is deterministic,
plain AGILE and surrogate-guided AGILE run end to end through the C ABI, and
the trained surrogate predicts full-fidelity losses better than the
low-fidelity loss it starts from -- the gain of the network over the same
schedule without it."""
import math

import numpy as np
import pytest

import spires_b200 as sp
from spires_b200 import search as S

pytestmark = pytest.mark.gpu

SPACE = S.Space(n_range=(100, 600))
RUNGS = (200, 800, 3200)


@pytest.fixture(scope="module")
def task():
    return S.Task(length=3200, val=500, washout=100)


def test_evaluator_is_deterministic(task):
    th = np.random.default_rng(3).uniform(0, 1, (12, S.DIM))
    a = S.Evaluator(SPACE, task, seed=1).evaluate(th, RUNGS[0], np.arange(12))
    b = S.Evaluator(SPACE, task, seed=1).evaluate(th, RUNGS[0], np.arange(12))
    assert np.array_equal(a, b)
    assert np.all(np.isfinite(a)) and np.all(a <= S.FAIL_LOSS)
    # the same point keeps its reservoir across fidelities: longer training
    # cannot make every candidate worse
    c = S.Evaluator(SPACE, task, seed=1).evaluate(th, RUNGS[-1], np.arange(12))
    assert np.median(c) <= np.median(a) + 0.5


def test_network_beats_low_fidelity_as_predictor(task):
    ev = S.Evaluator(SPACE, task, seed=2)
    rng = np.random.default_rng(5)
    th = rng.uniform(0, 1, (160, S.DIM))
    lo = ev.evaluate(th, RUNGS[0], np.arange(160))
    full = ev.evaluate(th, RUNGS[-1], np.arange(160))
    X = np.concatenate([SPACE.features(th), lo[:, None]], axis=1).astype(np.float32)
    net = sp.Surrogate(seed=0)
    net.train(X[:120], full[:120].astype(np.float32), epochs=300, batch=64, lr=1e-3, seed=0)
    m, v = net.predict(X[120:], bf16=True)
    rmse_net = float(np.sqrt(np.mean((m - full[120:]) ** 2)))
    rmse_low = float(np.sqrt(np.mean((lo[120:] - full[120:]) ** 2)))
    assert rmse_net < rmse_low, (rmse_net, rmse_low)
    assert np.all(np.isfinite(v))


def test_searches_run_and_surrogate_helps(task):
    kw = dict(chains=8, rungs=RUNGS, max_points=256, waves=4, seed=0)
    ev1 = S.Evaluator(SPACE, task, seed=1)
    with_net = S.surrogate_agile(ev1, **kw)
    ev2 = S.Evaluator(SPACE, task, seed=1)
    without = S.surrogate_agile(ev2, use_surrogate=False, **kw)
    ev3 = S.Evaluator(SPACE, task, seed=1)
    plain = S.plain_agile(ev3, chains=8, T=RUNGS[-1], seed=0, max_points=256)
    for r in (with_net, without, plain):
        assert math.isfinite(r.best_loss) and r.best_theta is not None
        assert r.history and all(b1 >= b2 for (_, b1), (_, b2) in zip(r.history, r.history[1:]))
    # the low-fidelity schedule simulates far fewer neuron-steps than plain AGILE
    assert ev1.stats.neuron_steps < 0.5 * ev3.stats.neuron_steps
    # the network-guided schedule finds at least as good a reservoir as the
    # same schedule ranked by the low-fidelity loss alone
    assert with_net.best_loss <= without.best_loss + 1e-12
    assert with_net.extra["tuples"] > 0 and without.extra["tuples"] == 0


def test_prescreen_skips_points_and_still_searches(task):
    """With the hyper-parameter pre-screen, part of each round's asked points
    is told the network's prediction without being built or simulated; the
    search still ends with a scored best point, and the low-fidelity
    simulations are fewer than without the pre-screen."""
    kw = dict(chains=8, rungs=RUNGS, max_points=256, waves=4, seed=0)
    ev1 = S.Evaluator(SPACE, task, seed=1)
    pre = S.surrogate_agile(ev1, prescreen=0.4, **kw)
    ev2 = S.Evaluator(SPACE, task, seed=1)
    full = S.surrogate_agile(ev2, **kw)
    assert math.isfinite(pre.best_loss) and pre.best_theta is not None
    assert pre.extra["screened_out"] > 0 and full.extra["screened_out"] == 0
    assert pre.extra["points"] == full.extra["points"]
    assert ev1.stats.neuron_steps < ev2.stats.neuron_steps
