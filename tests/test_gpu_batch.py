"""Batched multi-reservoir path: every instance of a batch of uneven
reservoirs (size, model, ring length, topology, series length, inputs) must
reproduce, bit for bit, the spike raster and final states of the same
reservoir created and run on its own -- and through it the oracle.

All calls go through the C ABI of libspires.so."""
import numpy as np
import pytest

import spires_b200 as sp
from tests import _oracle as O

pytestmark = pytest.mark.gpu


def gl_params(alpha, L):
    # [V_th, V_reset, V_rest, tau_m, alpha, T_mem, bias, t_ref] at dt = 1
    return (1.0, 0.0, 0.0, 20.0, alpha, float(L), 0.1, 2.0)


def mixed_batch(count, seed, n_lo=60, n_hi=3000, t_lo=40, t_hi=300):
    """Uneven instances in the spirit of a hyper-parameter sweep."""
    rng = np.random.default_rng(seed)
    cfgs, seeds, us = [], [], []
    topos = [sp.CONN_RANDOM, sp.CONN_SMALL_WORLD, sp.CONN_SCALE_FREE]
    for k in range(count):
        n = int(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi))))
        din = int(rng.integers(1, 4))
        topo = topos[k % 3]
        conn = float(rng.uniform(0.02, 0.2)) if topo == sp.CONN_RANDOM else 6.0 / (n - 1)
        if k % 2 == 0:
            L = int(rng.choice([16, 64, 128, 256]))
            cfg = sp.make_config(n, din, 2, rho=float(rng.uniform(0.5, 1.5)), ei=0.5,
                                 gamma=float(rng.uniform(0.5, 2.0)), conn=conn, topo=topo,
                                 neuron=sp.FLIF_GL,
                                 nparams=gl_params(float(rng.uniform(0.3, 1.0)), L))
        else:
            cfg = sp.make_config(n, din, 2, rho=float(rng.uniform(0.5, 1.5)), ei=0.5,
                                 gamma=float(rng.uniform(0.5, 2.0)), conn=conn, topo=topo,
                                 neuron=sp.LIF_DISCRETE, nparams=(0.0, 1.0, 0.1, 0.05))
        cfgs.append(cfg)
        seeds.append(int(rng.integers(1, 2**31 - 1)))
        T = int(rng.integers(t_lo, t_hi))
        us.append(rng.uniform(-1.0, 1.5, size=(T, din)))
    return cfgs, seeds, us


def same_bits(a, b):
    return np.array_equal(np.asarray(a).view(np.uint64), np.asarray(b).view(np.uint64))


def solo(cfg, seed, u):
    r = sp.Reservoir(cfg, seed=seed)
    _, R, _ = r.run_record(u, phi=False)
    V = r.state()
    r.close()
    return R, V


def test_batch_matches_single_reservoirs():
    cfgs, seeds, us = mixed_batch(14, seed=11)
    b = sp.Batch(cfgs, seeds)
    R, V, ms = b.run(us)
    assert ms > 0.0
    spiking = 0
    for k, (cfg, s, u) in enumerate(zip(cfgs, seeds, us)):
        R1, V1 = solo(cfg, s, u)
        bad = np.nonzero((R[k] != R1).any(axis=1))[0]
        assert bad.size == 0, f"instance {k}: raster differs first at step {bad[0]}"
        assert same_bits(V[k], V1), f"instance {k}: final states differ"
        spiking += int(np.unpackbits(R1.view(np.uint8)).sum() > 0)
    assert spiking >= 4  # the comparison is not only over silent rasters
    info = b.info()
    assert info["groups"] >= 2 and info["ctas"] >= info["groups"]
    b.close()


def test_batch_matches_oracle():
    cfgs, seeds, us = mixed_batch(4, seed=5, n_hi=400, t_hi=120)
    b = sp.Batch(cfgs, seeds)
    R, V, _ = b.run(us)
    for k, (cfg, s, u) in enumerate(zip(cfgs, seeds, us)):
        orc = O.Oracle(cfg, sp.HostModel(cfg, seed=s))
        phi_o, ras_o, _ = orc.run(u, y=False)
        ras = sp.unpack_raster(R[k], cfg.num_neurons)
        assert np.array_equal(ras, ras_o), f"instance {k}: raster differs from the oracle"
        assert same_bits(V[k], phi_o[-1]), f"instance {k}: states differ from the oracle"
    b.close()


def test_batch_repeat_replays_graph_and_is_deterministic():
    cfgs, seeds, us = mixed_batch(6, seed=21)
    b = sp.Batch(cfgs, seeds)
    R1, V1, _ = b.run(us)
    R2, V2, _ = b.run(us)
    assert b.info()["graph"] in (1, -1)
    for k in range(len(cfgs)):
        assert np.array_equal(R1[k], R2[k])
        assert same_bits(V1[k], V2[k])
    # other series lengths re-plan the schedule
    us3 = [u[: max(1, u.shape[0] // 2)] for u in us]
    R3, _, _ = b.run(us3)
    for k in range(len(cfgs)):
        assert np.array_equal(R3[k], R1[k][: us3[k].shape[0]])
    b.close()


def test_batch_zero_input_and_zero_length():
    cfgs, seeds, us = mixed_batch(3, seed=8, t_hi=80)
    b = sp.Batch(cfgs, seeds)
    T = [us[0].shape[0], 0, us[2].shape[0]]
    R, V, _ = b.run(None, T=T)
    for k in (0, 2):
        r = sp.Reservoir(cfgs[k], seed=seeds[k])
        _, R1, _ = r.run_record(np.zeros((T[k], cfgs[k].num_inputs)), phi=False)
        V1 = r.state()
        r.close()
        assert np.array_equal(R[k], R1)
        assert same_bits(V[k], V1)
    assert R[1].shape[0] == 0
    b.close()


def test_batch_ridge_and_predict_match_single():
    cfgs, seeds, us = mixed_batch(5, seed=31, n_hi=800, t_lo=150, t_hi=260)
    rng = np.random.default_rng(4)
    ys = [rng.standard_normal((u.shape[0], 2)) for u in us]
    b = sp.Batch(cfgs, seeds)
    W, ms = b.train_ridge(us, ys, 1e-4, washout=20)
    Yb, _ = b.predict(us)
    for k, (cfg, s, u) in enumerate(zip(cfgs, seeds, us)):
        r = sp.Reservoir(cfg, seed=s)
        o = sp.RidgeOpts(0, 30, 1e-13, 20)
        rep = sp.RidgeReport()
        st = r.lib.spires_ext_train_ridge(r.h, sp.dptr(u), sp.dptr(ys[k]), u.shape[0], 1e-4,
                                          sp.C.byref(o), sp.C.byref(rep))
        assert st == sp.SPIRES_OK
        W1 = r.readout()
        assert same_bits(W[k], W1), f"instance {k}: W_out differs"
        r.reset()
        Y1 = r.run(u)
        r.close()
        assert same_bits(Yb[k][:, :2], Y1), f"instance {k}: readouts differ"
    b.close()


def test_batch_rejects_unsupported_models():
    cfg = sp.make_config(64, 1, 1, neuron=sp.FLIF_CAPUTO,
                         nparams=O.NEURON_PARAMS[sp.FLIF_CAPUTO])
    with pytest.raises(RuntimeError):
        sp.Batch([cfg], [1])
    cfg2 = sp.make_config(64, 1, 1, neuron=sp.LIF_DISCRETE, synapse=sp.SYN_PSC_HOM,
                          sparams=(5.0,))
    with pytest.raises(RuntimeError):
        sp.Batch([cfg2], [1])


def test_fit_predict_equals_train_then_predict():
    cfgs, seeds, us = mixed_batch(4, seed=41, n_hi=600, t_lo=200, t_hi=300)
    rng = np.random.default_rng(2)
    ys = [rng.standard_normal((u.shape[0], 2)) for u in us]
    T_fit = [int(0.7 * u.shape[0]) for u in us]
    b = sp.Batch(cfgs, seeds)
    Y, _ = b.fit_predict(us, ys, T_fit, 1e-3, washout=10)
    b2 = sp.Batch(cfgs, seeds)
    b2.train_ridge([u[:t] for u, t in zip(us, T_fit)], [y[:t] for y, t in zip(ys, T_fit)], 1e-3,
                   washout=10)
    Y2, _ = b2.predict(us)
    for k in range(len(cfgs)):
        assert same_bits(Y[k][:, :2], Y2[k][:, :2]), f"instance {k}"


def test_autotuned_schedule_keeps_results():
    """spires_ext_batch_autotune times every schedule family and grid size on
    a sample of the series and keeps the fastest; whichever it keeps, every
    instance's raster and final state stay bit-identical to the same
    reservoir run on its own."""
    cfgs, seeds, us = mixed_batch(12, seed=77)
    b = sp.Batch(cfgs, seeds)
    sample = [u[:30] for u in us]
    tuned = b.autotune(sample)
    assert 0 <= tuned["schedule"] <= 3 and tuned["ctas"] > 0 and tuned["ms"] > 0
    R, V, _ = b.run(us)
    assert b.info()["ctas"] == tuned["ctas"]
    b.close()
    for k in range(len(cfgs)):
        Rs, Vs = solo(cfgs[k], seeds[k], us[k])
        assert np.array_equal(R[k], Rs), k
        assert same_bits(V[k], Vs), k


def test_batch_runs_after_a_smaller_batch_was_built():
    """The batch kernel's shared-memory limit is one attribute for the whole
    process. A batch with long rings (large shared memory) must still launch
    after a second batch with short rings (less shared memory, still above the
    48 KB default) was built, and re-plan for new
    series lengths (a search builds the next chunk's batch on another thread
    while the current one runs)."""
    big_cfg = sp.make_config(1500, 1, 1, rho=0.9, ei=0.5, gamma=1.0, conn=0.05,
                             topo=sp.CONN_RANDOM, neuron=sp.FLIF_GL,
                             nparams=gl_params(0.6, 1024))
    small_cfg = sp.make_config(300, 1, 1, rho=0.9, ei=0.5, gamma=1.0, conn=0.05,
                               topo=sp.CONN_RANDOM, neuron=sp.FLIF_GL,
                               nparams=gl_params(0.6, 128))
    rng = np.random.default_rng(5)
    big = sp.Batch([big_cfg, big_cfg], [11, 12])
    small = sp.Batch([small_cfg], [13])
    try:
        for T in (60, 140):
            us = [rng.uniform(-1.0, 1.5, size=(T, 1)) for _ in range(2)]
            R, V, _ = big.run(us)
            for k, seed in enumerate((11, 12)):
                Rs, Vs = solo(big_cfg, seed, us[k])
                assert np.array_equal(R[k], Rs)
                assert same_bits(V[k], Vs)
        small.run([rng.uniform(-1.0, 1.5, size=(50, 1))])
    finally:
        big.close()
        small.close()
