"""GPU parity: the CUDA step kernels against the oracle (and the compiled
reference when present), bit for bit on states and spike rasters.

All calls go through the C ABI of libspires.so."""
import numpy as np
import pytest

import spires_b200 as sp
from tests import _oracle as O

pytestmark = pytest.mark.gpu

NEURONS = [sp.LIF_DISCRETE, sp.LIF_BIO, sp.FLIF_CAPUTO, sp.FLIF_GL, sp.FLIF_DIFFUSIVE]
SYNAPSES = [sp.SYN_SIMPLE, sp.SYN_PSC_HOM, sp.SYN_PSC_HET, sp.SYN_FRAC, sp.SYN_FRAC_MEXP]


def make(neuron, synapse, n=96, din=2, dout=2, dt=1.0, topo=sp.CONN_RANDOM, conn=0.08,
         backend=0, gamma=1.2, rho=1.3, nparams=None):
    return sp.make_config(n, din, dout, rho=rho, ei=0.55, gamma=gamma, conn=conn, dt=dt,
                          topo=topo, neuron=neuron,
                          nparams=nparams or O.NEURON_PARAMS[neuron], synapse=synapse,
                          backend=backend, sparams=O.SYNAPSE_PARAMS[synapse])


def inputs(T, din, seed=3):
    return np.random.default_rng(seed).uniform(-1.0, 1.5, size=(T, din))


def same_bits(a, b):
    return np.array_equal(np.asarray(a).view(np.uint64), np.asarray(b).view(np.uint64))


def run_both(cfg, seed, T, launch=None, y=True):
    u = inputs(T, cfg.num_inputs)
    r = sp.Reservoir(cfg, seed=seed)
    if launch:
        assert r.set_launch(**launch) == sp.SPIRES_OK
    phi, R, Y = r.run_record(u, y=y)
    ras = sp.unpack_raster(R, r.n)
    r.close()
    orc = O.Oracle(cfg, sp.HostModel(cfg, seed=seed))
    phi_o, ras_o, Y_o = orc.run(u, y=y)
    return (phi, ras, Y), (phi_o, ras_o, Y_o), u


def assert_parity(mine, ref, dout):
    phi, ras, Y = mine
    phi_o, ras_o, Y_o = ref
    bad = np.nonzero((ras != ras_o).any(axis=1))[0]
    assert bad.size == 0, f"raster differs first at step {bad[0]}"
    assert same_bits(phi, phi_o), "states differ"
    if Y is not None:
        # readouts use a fixed parallel reduction: tolerance on |y - y_ref|
        Y = Y[:, :dout]
        Y_o = Y_o[:, :dout]
        scale = np.abs(phi_o).sum(axis=1, keepdims=True) + 1.0
        assert np.all(np.abs(Y - Y_o) <= 1e-12 * scale)


@pytest.mark.parametrize("neuron", NEURONS)
@pytest.mark.parametrize("synapse", SYNAPSES)
def test_models_bit_exact(neuron, synapse):
    cfg = make(neuron, synapse)
    mine, ref, _ = run_both(cfg, seed=11, T=80)
    assert_parity(mine, ref, 2)
    assert mine[1].mean() > 0.0


@pytest.mark.parametrize("n", [1, 31, 32, 33, 200, 1000])
def test_sizes_and_word_boundaries(n):
    cfg = make(sp.FLIF_GL, sp.SYN_SIMPLE, n=n, conn=min(0.5, 8.0 / max(n, 2)))
    mine, ref, _ = run_both(cfg, seed=2, T=50)
    assert_parity(mine, ref, 2)


@pytest.mark.parametrize("ctas,warps", [(1, 32), (2, 16), (5, 7), (32, 1)])
def test_launch_shapes_identical(ctas, warps):
    cfg = make(sp.FLIF_GL, sp.SYN_PSC_HET, n=1000, conn=0.02)
    mine, ref, _ = run_both(cfg, seed=8, T=40, launch=dict(ctas=ctas, warps_max=warps))
    assert_parity(mine, ref, 2)


@pytest.mark.parametrize("neuron", [sp.LIF_BIO, sp.FLIF_GL, sp.FLIF_CAPUTO])
def test_micro_steps(neuron):
    cfg = make(neuron, sp.SYN_FRAC, dt=0.25)
    mine, ref, _ = run_both(cfg, seed=5, T=30)
    assert_parity(mine, ref, 2)


@pytest.mark.parametrize("topo,conn,backend", [(sp.CONN_SMALL_WORLD, 10 / 399, 0),
                                               (sp.CONN_SCALE_FREE, 5 / 399, 0),
                                               (sp.CONN_RANDOM, 0.1, 1)])
def test_topologies(topo, conn, backend):
    cfg = make(sp.FLIF_GL, sp.SYN_SIMPLE, n=400, topo=topo, conn=conn, backend=backend)
    mine, ref, _ = run_both(cfg, seed=21, T=120)
    assert_parity(mine, ref, 2)


def test_public_api_step_read_matches_oracle():
    """spires_step / read_state / read_spike_state / compute_output, one call per step."""
    cfg = make(sp.FLIF_GL, sp.SYN_PSC_HOM, n=150)
    u = inputs(40, 2)
    r = sp.Reservoir(cfg, seed=31)
    orc = O.Oracle(cfg, sp.HostModel(cfg, seed=31))
    phi_o, ras_o, Y_o = orc.run(u, y=True)
    for t in range(40):
        r.step(u[t])
        assert same_bits(r.state(), phi_o[t])
        assert np.array_equal(r.spikes(), ras_o[t].astype(np.float64))
        y = r.output()
        assert np.all(np.abs(y - Y_o[t, :2]) <= 1e-12 * (np.abs(phi_o[t]).sum() + 1))
    # spires_run continues from the same state and returns the same readouts
    u2 = inputs(25, 2, seed=9)
    Yr = r.run(u2)
    _, _, Y2 = orc.run(u2, y=True)
    assert np.all(np.abs(Yr - Y2[:, :2]) <= 1e-12 * 1e3)
    r.close()


def test_null_input_is_zero_vector():
    cfg = make(sp.FLIF_GL, sp.SYN_SIMPLE, n=64, gamma=1.0)
    r = sp.Reservoir(cfg, seed=3)
    for _ in range(5):
        r.step(None)
    v1 = r.state()
    r.reset()
    for _ in range(5):
        r.step(np.zeros(2))
    assert same_bits(v1, r.state())
    r.close()


def test_reset_keeps_synapse_state_like_reference():
    """reset re-initialises neurons only; PSC traces carry over (reference quirk)."""
    cfg = make(sp.FLIF_GL, sp.SYN_PSC_HOM, n=120)
    u = inputs(30, 2)
    r = sp.Reservoir(cfg, seed=6)
    r.run_record(u)
    r.reset()
    phi, R, _ = r.run_record(u)
    r.close()
    orc = O.Oracle(cfg, sp.HostModel(cfg, seed=6))
    orc.run(u)
    orc.reset()
    phi_o, ras_o, _ = orc.run(u)
    assert same_bits(phi, phi_o)
    assert np.array_equal(sp.unpack_raster(R, 120), ras_o)


@pytest.mark.skipif(not O.have_ref(), reason="reference build absent")
def test_against_compiled_reference_directly():
    cfg = make(sp.FLIF_GL, sp.SYN_PSC_HET, n=128)
    u = inputs(50, 2)
    phi_r, ras_r = O.ref_trajectory(cfg, 77, u)
    r = sp.Reservoir(cfg, seed=77)
    phi, R, _ = r.run_record(u)
    r.close()
    assert same_bits(phi, phi_r)
    assert np.array_equal(sp.unpack_raster(R, 128), ras_r)


def test_flif_gl_n4000_l512_small_world():
    """FLIF_GL N=4000, L=512, Watts-Strogatz k=10, rho=0.95 (the FP64
    fractional-order configuration), 600 steps bit-exact against the oracle:
    the ring wraps once, so every lag of the history sum is exercised."""
    params = (1.0, 0.0, 0.0, 20.0, 0.7, 512.0, 0.1, 2.0)
    cfg = sp.make_config(4000, 1, 1, rho=0.95, ei=0.5, gamma=0.5, conn=10 / 3999, dt=1.0,
                         topo=sp.CONN_SMALL_WORLD, neuron=sp.FLIF_GL, nparams=params)
    from spires_b200 import datasets
    x = datasets.mackey_glass(601, seed=0)
    u = x[:600, None]
    r = sp.Reservoir(cfg, seed=42)
    phi, R, _ = r.run_record(u)
    r.close()
    orc = O.Oracle(cfg, sp.HostModel(cfg, seed=42))
    phi_o, ras_o, _ = orc.run(u)
    ras = sp.unpack_raster(R, 4000)
    assert ras.mean() > 0.01
    assert np.array_equal(ras, ras_o)
    assert same_bits(phi, phi_o)


GL_L = lambda L: (1.0, 0.0, 0.0, 20.0, 0.7, float(L), 0.1, 2.0)


@pytest.mark.parametrize("L", [3, 8, 33, 200])
@pytest.mark.parametrize("shape", [dict(ctas=1, warps_max=8, rows=16, stages=2),
                                   dict(ctas=4, warps_max=2, rows=3, stages=3),
                                   dict(ctas=8, warps_max=1, rows=1, stages=4),
                                   dict(ctas=2, warps_max=4, rows=16, stages=8),
                                   dict(ctas=4, warps_max=2, rows=8, stages=5),
                                   dict(ctas=1, warps_max=8, rows=32, stages=2)])
def test_flif_gl_bulk_copy_pipeline(L, shape):
    """The bulk-copy ring pipeline (variant 1) gives the bits of the oracle for
    ring lengths shorter and longer than its depth, during ramp-up (step < L)
    and after the ring wraps."""
    cfg = make(sp.FLIF_GL, sp.SYN_SIMPLE, n=250, conn=0.03, nparams=GL_L(L))
    mine, ref, _ = run_both(cfg, seed=13, T=2 * L + 40, launch=dict(variant=1, **shape))
    assert_parity(mine, ref, 2)


@pytest.mark.parametrize("synapse", SYNAPSES)
def test_flif_gl_pipeline_all_synapses(synapse):
    cfg = make(sp.FLIF_GL, synapse, n=300, conn=0.03, nparams=GL_L(96))
    a, ref, _ = run_both(cfg, seed=17, T=150, launch=dict(variant=1, ctas=3, warps_max=4,
                                                          rows=16, stages=4))
    assert_parity(a, ref, 2)
    b, _, _ = run_both(cfg, seed=17, T=150, launch=dict(variant=0, ctas=3, warps_max=4))
    assert same_bits(a[0], b[0])


def test_flif_gl_pipeline_chunked_runs_continue():
    """Several launches in a row (state carried in HBM between them) equal one."""
    cfg = make(sp.FLIF_GL, sp.SYN_SIMPLE, n=500, conn=0.02, nparams=GL_L(128))
    u = inputs(300, 2)
    r = sp.Reservoir(cfg, seed=19)
    parts = [r.run_record(u[a:b])[0] for a, b in [(0, 1), (1, 50), (50, 129), (129, 300)]]
    r.close()
    phi = np.concatenate(parts)
    phi_o, _, _ = O.Oracle(cfg, sp.HostModel(cfg, seed=19)).run(u)
    assert same_bits(phi, phi_o)


@pytest.mark.parametrize("neuron,L", [(sp.FLIF_GL, 256), (sp.LIF_DISCRETE, 1)])
def test_autotune_keeps_state_and_results(neuron, L):
    """spires_ext_autotune times launch shapes from a saved state and restores
    it: a run continued after tuning equals an untuned run bit for bit."""
    nparams = GL_L(L) if neuron == sp.FLIF_GL else O.NEURON_PARAMS[neuron]
    cfg = make(neuron, sp.SYN_SIMPLE, n=3000, conn=0.003, nparams=nparams)
    u = inputs(200, 2)
    a = sp.Reservoir(cfg, seed=23)
    pa1, _, _ = a.run_record(u[:100])
    assert a.lib.spires_ext_autotune(a.h, 32) == sp.SPIRES_OK
    pa2, _, _ = a.run_record(u[100:])
    a.close()
    b = sp.Reservoir(cfg, seed=23)
    pb, _, _ = b.run_record(u)
    b.close()
    assert same_bits(np.concatenate([pa1, pa2]), pb)
