"""GPU readouts against the oracle (and the compiled reference when present):
ridge (src/reservoir.c:573-679), RLS (:681-767), the online delta rule
(:244-280), coarse-graining (:782-967) and the readout itself (:169-192).

Readout solves are floating-point reductions in a different order than the
reference (blocked Cholesky + refinement instead of one LU per output), so they
are compared with tolerances stated per test; states feeding them are
bit-identical (tests/test_gpu_parity.py)."""
import ctypes as C

import numpy as np
import pytest

import spires_b200 as sp
from tests import _oracle as O

pytestmark = pytest.mark.gpu

GL = (1.0, 0.0, 0.0, 20.0, 0.7, 64.0, 0.1, 2.0)


def cfg_gl(n=200, din=2, dout=3, conn=0.04, topo=sp.CONN_SCALE_FREE, synapse=sp.SYN_SIMPLE):
    return sp.make_config(n, din, dout, rho=1.2, ei=0.55, gamma=1.2, conn=conn, topo=topo,
                          neuron=sp.FLIF_GL, nparams=GL, synapse=synapse,
                          sparams=O.SYNAPSE_PARAMS[synapse])


def data(T, din, dout, seed=0):
    rng = np.random.default_rng(seed)
    u = rng.uniform(-1.0, 1.5, size=(T, din))
    y = np.stack([np.sin(0.05 * np.arange(T) * (o + 1)) for o in range(dout)], axis=1)
    y = y + 0.1 * rng.standard_normal((T, dout))
    return u, np.ascontiguousarray(y)


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("lam", [1e-2, 1e-6])
def test_ridge_matches_fp64_oracle(lam):
    cfg = cfg_gl()
    u, y = data(500, 2, 3)
    r = sp.Reservoir(cfg, seed=3)
    r.train_ridge(u, y, lam)
    W = r.readout()
    r.close()
    orc = O.Oracle(cfg, sp.HostModel(cfg, seed=3))
    phi, _, _ = orc.run(u)
    Wo = O.oracle_ridge(phi, y, lam)
    # tolerance: the solution's sensitivity is cond(A) * eps; both solvers are
    # backward stable, so compare the fitted outputs tightly and W loosely
    assert rel(phi @ W.T, phi @ Wo.T) < 1e-9
    assert rel(W, Wo) < (1e-9 if lam >= 1e-2 else 1e-5)


@pytest.mark.skipif(not O.have_ref(), reason="reference build absent")
def test_ridge_matches_compiled_reference():
    cfg = cfg_gl(n=150)
    u, y = data(400, 2, 3, seed=4)
    r = sp.Reservoir(cfg, seed=8)
    r.train_ridge(u, y, 1e-3)
    W = r.readout()
    r.close()
    ref = sp.Reservoir(cfg, lib=O.ref_lib(), seed=8)
    ref.train_ridge(u, y, 1e-3)
    Wr = ref.readout()
    ref.close()
    assert rel(W, Wr) < 1e-9


def test_ridge_washout_and_report():
    cfg = cfg_gl()
    u, y = data(600, 2, 3, seed=5)
    r = sp.Reservoir(cfg, seed=3)
    opts = sp.RidgeOpts(0, 30, 1e-13, 100)
    rep = sp.RidgeReport()
    assert r.lib.spires_ext_train_ridge(r.h, sp.dptr(u), sp.dptr(y), 600, 1e-4, C.byref(opts),
                                        C.byref(rep)) == sp.SPIRES_OK
    W = r.readout()
    r.close()
    orc = O.Oracle(cfg, sp.HostModel(cfg, seed=3))
    phi, _, _ = orc.run(u)
    Wo = O.oracle_ridge(phi, y, 1e-4, washout=100)
    assert rel(phi[100:] @ W.T, phi[100:] @ Wo.T) < 1e-9
    assert rep.rel_residual < 1e-10
    assert rep.gram_mode_used == 0


def test_ridge_singular_system_keeps_going():
    """lambda = 0 with fewer samples than neurons: a singular system. The call
    returns OK as the reference does (it only prints a warning)."""
    cfg = cfg_gl(n=120)
    u, y = data(40, 2, 3, seed=6)
    r = sp.Reservoir(cfg, seed=2)
    r.train_ridge(u, y, 0.0)
    r.close()


def test_rls_matches_oracle():
    cfg = cfg_gl(n=80, conn=0.06)
    u, y = data(60, 2, 3, seed=7)
    r = sp.Reservoir(cfg, seed=12)
    r.train_rls(u, y, 1.0, 0.999)
    W = r.readout()
    r.close()
    orc = O.Oracle(cfg, sp.HostModel(cfg, seed=12))
    Wo = orc.train_rls(u, y, 1.0, 0.999)
    assert rel(W, Wo) < 1e-8


def test_online_rule_matches_oracle():
    cfg = cfg_gl(n=100)
    u, y = data(50, 2, 3, seed=9)
    hm = sp.HostModel(cfg, seed=21)
    r = sp.Reservoir(cfg, seed=21)
    orc = O.Oracle(cfg, hm)
    Wo = hm.w_out().copy()
    for t in range(50):
        r.step(u[t])
        orc.step(u[t])
        r.train_online(y[t], 0.01)
        orc.train_online(y[t], 0.01, Wo)
    assert rel(r.readout(), Wo) < 1e-12
    r.close()


def test_run_and_compute_output_agree_bitwise():
    """spires_run and spires_step + spires_compute_output use one readout
    reduction, so they return the same bits."""
    cfg = cfg_gl(n=300)
    u, _ = data(30, 2, 3)
    a = sp.Reservoir(cfg, seed=5)
    Ya = a.run(u)
    a.close()
    b = sp.Reservoir(cfg, seed=5)
    Yb = []
    for t in range(30):
        b.step(u[t])
        Yb.append(b.output())
    b.close()
    assert np.array_equal(Ya, np.array(Yb))


# ------------------------------------------------------------ coarse grain

def coarse_grain_restated(W, Win, Wout, V, thr):
    """src/reservoir.c:782-967 in plain Python (small n only)."""
    n = W.shape[0]
    W = W.copy(); Win = Win.copy(); Wout = Wout.copy(); V = V.copy()
    alive = np.ones(n, bool)
    merged = True
    while merged:
        merged = False
        for i in range(n):
            for j in range(i + 1, n):
                if W[i, j] <= thr and W[j, i] <= thr:
                    continue
                merged = True
                V[i] = (V[i] + V[j]) / 2.0
                V[j] = 0.0
                alive[j] = False
                for k in range(n):
                    if k == i or k == j:
                        continue
                    a, b = W[i, k], W[j, k]
                    nw = a + b if a * b == 0.0 else (a + b) / 2.0
                    W[i, k] = nw
                    W[k, i] = nw
                for k in range(Win.shape[1]):
                    a, b = Win[i, k], Win[j, k]
                    Win[i, k] = a + b if a * b == 0.0 else (a + b) / 2.0
                    Win[j, k] = 0.0
                Wout[:, i] += Wout[:, j]
                Wout[:, j] = 0.0
                W[j, :] = 0.0
                W[:, j] = 0.0
    idx = np.nonzero(alive)[0]
    return W[np.ix_(idx, idx)], Win[idx], Wout[:, idx], V[idx]


def test_coarse_grain_matches_restatement():
    cfg = cfg_gl(n=40, conn=0.15, topo=sp.CONN_RANDOM)
    u, _ = data(20, 2, 3)
    r = sp.Reservoir(cfg, seed=14)
    for t in range(20):
        r.step(u[t])
    W, Win, Wout, V = r.weights(), r.w_in(), r.readout(), r.state()
    h = C.c_void_p()
    assert r.lib.spires_coarse_grain(r.h, 0.05, C.byref(h)) == sp.SPIRES_OK
    Wc, Winc, Woutc, Vc = coarse_grain_restated(W, Win, Wout, V, 0.05)
    m = Wc.shape[0]
    assert r.lib.spires_num_neurons(h) == m
    nw = np.empty(m * m)
    r.lib.spires_read_weights(h, sp.dptr(nw))
    assert np.array_equal(nw.reshape(m, m), Wc)
    no = np.empty(3 * m)
    r.lib.spires_read_readout(h, sp.dptr(no))
    assert np.array_equal(no.reshape(3, m), Woutc)
    ns = np.empty(m)
    r.lib.spires_read_reservoir_state(h, sp.dptr(ns))
    assert np.array_equal(ns, Vc)
    wi = np.empty(m * 2)
    r.lib.spires_ext_read_w_in(h, sp.dptr(wi))
    assert np.array_equal(wi.reshape(m, 2), Winc)
    # the coarse reservoir steps like any other
    for t in range(5):
        r.lib.spires_step(h, sp.dptr(np.ascontiguousarray(u[t])))
    r.lib.spires_reservoir_destroy(h)
    # thresholds below zero (or NaN) would merge forever: refused
    h2 = C.c_void_p()
    for thr in (-0.5, float("nan")):
        assert r.lib.spires_coarse_grain(r.h, thr, C.byref(h2)) == sp.SPIRES_ERR_INVALID_ARG
    r.close()


@pytest.mark.parametrize("lam", [1e-2, 1e-5])
def test_ridge_dual_form_when_rows_are_few(lam):
    """Fewer fitted rows than N/2: the dual form solves the same ridge."""
    cfg = cfg_gl(n=700, conn=0.02)
    u, y = data(300, 2, 3, seed=9)
    r = sp.Reservoir(cfg, seed=5)
    opts = sp.RidgeOpts(0, 30, 1e-13, 20)
    rep = sp.RidgeReport()
    assert r.lib.spires_ext_train_ridge(r.h, sp.dptr(u), sp.dptr(y), 300, lam, C.byref(opts),
                                        C.byref(rep)) == sp.SPIRES_OK
    W = r.readout()
    r.close()
    assert rep.dual == 1
    orc = O.Oracle(cfg, sp.HostModel(cfg, seed=5))
    phi, _, _ = orc.run(u)
    Wo = O.oracle_ridge(phi, y, lam, washout=20)
    assert rel(phi[20:] @ W.T, phi[20:] @ Wo.T) < 1e-8
    assert rel(W, Wo) < (1e-6 if lam >= 1e-2 else 1e-3)
    assert rep.rel_residual < 1e-8


def test_ridge_more_than_sixteen_outputs():
    """21 outputs, as many as a caller likes in the reference: solved 16 at a
    time over the one system matrix, the FP64 oracle's solution for all of
    them, through the reservoir and through ridge_fit on host states."""
    cfg = cfg_gl(dout=21)
    u, y = data(500, 2, 21, seed=9)
    r = sp.Reservoir(cfg, seed=3)
    r.train_ridge(u, y, 1e-2)
    W = r.readout()
    r.close()
    orc = O.Oracle(cfg, sp.HostModel(cfg, seed=3))
    phi, _, _ = orc.run(u)
    Wo = O.oracle_ridge(phi, y, 1e-2)
    assert W.shape == (21, cfg.num_neurons)
    assert rel(phi @ W.T, phi @ Wo.T) < 1e-9
    assert rel(W, Wo) < 1e-9
    W2, _ = sp.ridge_fit(phi, y, 1e-2)
    assert rel(W2, Wo) < 1e-9
