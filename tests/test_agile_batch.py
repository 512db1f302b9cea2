"""AGILE in ask/tell form: chains advanced in lockstep visit exactly the points
that the sequential optimiser (spires_ext_agile_minimize, itself pinned to the
reference's agile_optimize) visits with the same options and seed. CPU only."""
import ctypes as C

import numpy as np
import pytest

import spires_b200 as sp


def objective(x):
    v = sum(100.0 * (x[i + 1] - x[i] ** 2) ** 2 + (1.0 - x[i]) ** 2 for i in range(len(x) - 1))
    return float(v + 0.3 * np.sin(3.0 * x).sum())


def sequential(th0, lo, hi, opts):
    dim = len(th0)
    log = []

    def f(theta, d, ctx):
        x = np.ctypeslib.as_array(theta, shape=(d,)).copy()
        log.append(x)
        return objective(x)
    cb = sp.LOSS_FN(f)
    best = (C.c_double * dim)()
    rep = sp.AgileReport()
    st = sp.load().spires_ext_agile_minimize((C.c_double * dim)(*th0), (C.c_double * dim)(*lo),
                                             (C.c_double * dim)(*hi), dim, cb, None,
                                             C.byref(opts), best, C.byref(rep))
    assert st == 0
    return np.array(best[:]), rep, np.array(log)


@pytest.mark.parametrize("reflect", [0, 1])
def test_lockstep_chains_match_sequential(reflect):
    lib = sp.load()
    dim, chains = 4, 3
    rng = np.random.default_rng(5)
    th0 = rng.uniform(-1, 1, (chains, dim))
    lo = np.full(dim, -1.5)
    hi = np.full(dim, 1.5)
    seeds = (C.c_uint64 * chains)(0xA91E, 12345, 777)
    opts = sp.AgileOpts(1.3, 1e-3, 0.3, 12.0, 0.9, 1e-3, 40, 10, 1e-3, reflect, 0, 0)
    h = C.c_void_p()
    th0c = np.ascontiguousarray(th0)
    assert lib.spires_ext_agile_batch_create(chains, dim, sp.dptr(th0c), sp.dptr(lo), sp.dptr(hi),
                                             C.byref(opts), seeds, C.byref(h)) == 0
    pts = np.empty((2 * chains, dim))
    owner = (C.c_int * (2 * chains))()
    logs = [[] for _ in range(chains)]
    rounds = 0
    while True:
        n = lib.spires_ext_agile_batch_ask(h, sp.dptr(pts), owner)
        if n == 0:
            break
        losses = np.array([objective(pts[k]) for k in range(n)])
        for k in range(n):
            logs[owner[k]].append(pts[k].copy())
        assert lib.spires_ext_agile_batch_tell(h, sp.dptr(losses)) == 0
        rounds += 1
        assert rounds < 100000
    for k in range(chains):
        o = sp.AgileOpts(1.3, 1e-3, 0.3, 12.0, 0.9, 1e-3, 40, 10, 1e-3, reflect, seeds[k], 0)
        best, rep, log = sequential(th0[k], lo, hi, o)
        assert np.array_equal(np.array(logs[k]), log), f"chain {k}: evaluation sequence differs"
        b = np.empty(dim)
        r = sp.AgileReport()
        assert lib.spires_ext_agile_batch_best(h, k, sp.dptr(b), C.byref(r)) == 0
        assert np.array_equal(b, best)
        assert (r.best_loss, r.best_iter, r.total_evals, r.total_iters, r.exited_refinement) == \
            (rep.best_loss, rep.best_iter, rep.total_evals, rep.total_iters,
             rep.exited_refinement)
    lib.spires_ext_agile_batch_destroy(h)
