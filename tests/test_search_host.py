"""Host logic of the search and sweep drivers (no GPU): decoding of the
encoded hyper-parameters, surrogate features, seeded populations, task
series, and the classification data's class offsets."""
import math

import numpy as np

import spires_b200 as sp
from spires_b200 import datasets, search, sweep


def test_space_decode_bounds_and_snaps():
    sp_ = search.Space()
    lo = sp_.decode(np.zeros(search.DIM))
    hi = sp_.decode(np.ones(search.DIM))
    assert lo["n"] == 500 and hi["n"] == 8000
    assert lo["neuron"] == sp.LIF_DISCRETE and hi["neuron"] == sp.FLIF_GL
    assert lo["L"] == 128 and hi["L"] == 1024
    assert lo["topo"] == sp.CONN_RANDOM and hi["topo"] == sp.CONN_SCALE_FREE
    assert math.isclose(lo["lam"], 1e-8) and math.isclose(hi["lam"], 1.0)
    assert math.isclose(lo["gain"], 10 ** -2.5) and math.isclose(hi["gain"], 1.0)
    # out-of-box points are clipped, not extrapolated
    assert sp_.decode(np.full(search.DIM, 2.0))["n"] == 8000


def test_features_are_unit_box_and_snapped():
    sp_ = search.Space()
    th = np.random.default_rng(0).uniform(-0.2, 1.2, (50, search.DIM))
    f = sp_.features(th)
    assert f.shape == (50, search.DIM)
    assert f.min() >= 0.0 and f.max() <= 1.0
    assert set(np.unique(f[:, 1])) <= {0.0, 1.0}
    assert set(np.round(np.unique(f[:, 6]) * 2)) <= {0.0, 1.0, 2.0}


def test_config_carries_decoded_parameters():
    cfg, d = search.Space().config(np.full(search.DIM, 0.75))
    assert cfg.num_neurons == d["n"] and cfg.neuron_type == sp.FLIF_GL
    assert math.isclose(cfg.input_strength, d["gain"])
    p = np.ctypeslib.as_array(cfg.neuron_params, shape=(8,))
    assert p[4] == d["alpha"] and p[5] == float(d["L"])


def test_sweep_space_is_seeded():
    a = sweep.sweep_space(20, seed=3)
    b = sweep.sweep_space(20, seed=3)
    assert [(i.n, i.T, i.seed, i.topo) for i in a] == [(i.n, i.T, i.seed, i.topo) for i in b]
    assert all(500 <= i.n <= 8000 and 2000 <= i.T <= 10000 for i in a)
    assert all(0.02 <= i.conn <= 0.2 for i in a)


def test_task_series_shapes():
    t = search.Task(length=500, val=100, washout=50)
    u, y = t.series(300)
    assert u.shape == (400, 1) and y.shape == (400, 1)
    assert np.array_equal(u[1:, 0], y[:-1, 0])


def test_bursty_offsets_parameter():
    a, la = datasets.bursty_sinusoids(20, seed=1)
    b, lb = datasets.bursty_sinusoids(20, seed=1, offset_span=0.015)
    assert np.array_equal(la, lb) and all(np.array_equal(x, y) for x, y in zip(a, b))
    c, _ = datasets.bursty_sinusoids(20, seed=1, offset_span=0.05)
    assert not all(np.array_equal(x, y) for x, y in zip(a, c))


def test_search_result_time_to():
    r = search.SearchResult(-2.0, None, 10.0, 5, [(1.0, -1.0), (4.0, -1.5), (9.0, -2.0)])
    assert r.time_to(-1.2) == 4.0 and r.time_to(-3.0) is None
    assert math.isclose(r.best_nrmse, math.exp(-2.0))
