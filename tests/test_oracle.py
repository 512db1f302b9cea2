"""The oracle (C restatement, oracle/spires_oracle.c) reproduces the reference
compiled from source bit for bit: states and spike rasters after every
macro step, for every neuron x synapse model, both storage backends and
micro-stepping. CPU only."""
import numpy as np
import pytest

import spires_b200 as sp
from tests import _oracle as O

pytestmark = pytest.mark.skipif(not O.have_ref(), reason="reference build absent")

NEURONS = [sp.LIF_DISCRETE, sp.LIF_BIO, sp.FLIF_CAPUTO, sp.FLIF_GL, sp.FLIF_DIFFUSIVE]
SYNAPSES = [sp.SYN_SIMPLE, sp.SYN_PSC_HOM, sp.SYN_PSC_HET, sp.SYN_FRAC, sp.SYN_FRAC_MEXP]


def make(neuron, synapse, n=96, din=2, dt=1.0, topo=sp.CONN_RANDOM, conn=0.08, backend=0,
         gamma=1.2, rho=1.3):
    return sp.make_config(n, din, 2, rho=rho, ei=0.55, gamma=gamma, conn=conn, dt=dt,
                          topo=topo, neuron=neuron, nparams=O.NEURON_PARAMS[neuron],
                          synapse=synapse, backend=backend,
                          sparams=O.SYNAPSE_PARAMS[synapse])


def inputs(T, din, seed=3):
    rng = np.random.default_rng(seed)
    return rng.uniform(-1.0, 1.5, size=(T, din))


def check(cfg, seed, T=60):
    u = inputs(T, cfg.num_inputs)
    phi_r, ras_r = O.ref_trajectory(cfg, seed, u)
    hm = sp.HostModel(cfg, seed=seed)
    orc = O.Oracle(cfg, hm)
    phi_o, ras_o, _ = orc.run(u)
    assert np.array_equal(ras_r, ras_o), "spike rasters differ"
    assert np.array_equal(phi_r.view(np.uint64), phi_o.view(np.uint64)), "states differ"
    return ras_r.mean()


@pytest.mark.parametrize("neuron", NEURONS)
@pytest.mark.parametrize("synapse", SYNAPSES)
def test_oracle_matches_reference(neuron, synapse):
    rate = check(make(neuron, synapse), seed=11)
    assert rate > 0.0 or neuron == sp.FLIF_CAPUTO  # dynamics are exercised


@pytest.mark.parametrize("neuron", [sp.LIF_BIO, sp.FLIF_GL, sp.FLIF_CAPUTO])
def test_oracle_micro_steps(neuron):
    check(make(neuron, sp.SYN_PSC_HOM, dt=0.25), seed=5, T=30)


@pytest.mark.parametrize("topo,conn", [(sp.CONN_SMALL_WORLD, 6 / 95), (sp.CONN_SCALE_FREE, 3 / 95)])
@pytest.mark.parametrize("backend", [0, 1])
def test_oracle_topologies_backends(topo, conn, backend):
    check(make(sp.FLIF_GL, sp.SYN_SIMPLE, topo=topo, conn=conn, backend=backend), seed=9)


def test_oracle_readout_and_reset():
    cfg = make(sp.FLIF_GL, sp.SYN_SIMPLE)
    u = inputs(40, 2)
    r = sp.Reservoir(cfg, lib=O.ref_lib(), seed=4)
    Yr = r.run(u)
    r.reset()
    Yr2 = r.run(u)
    r.close()
    hm = sp.HostModel(cfg, seed=4)
    orc = O.Oracle(cfg, hm)
    _, _, Yo = orc.run(u, y=True)
    orc.reset()
    _, _, Yo2 = orc.run(u, y=True)
    assert np.array_equal(Yr, Yo)
    assert np.array_equal(Yr2, Yo2)


def test_oracle_matches_reference_randomised():
    """Randomised neuron x synapse x micro-stepping x topology x backend,
    with the fractional order and memory of FLIF_GL, the leak of LIF_DISCRETE
    and the input gain drawn too: the checker itself pinned beyond the grid."""
    rng = np.random.default_rng(77)
    for trial in range(12):
        neuron = NEURONS[int(rng.integers(0, len(NEURONS)))]
        synapse = SYNAPSES[int(rng.integers(0, len(SYNAPSES)))]
        params = list(O.NEURON_PARAMS[neuron])
        if neuron == sp.FLIF_GL:
            params[4] = float(rng.uniform(0.3, 1.0))
            params[5] = float(rng.choice([8.0, 33.0, 64.0]))
        if neuron == sp.LIF_DISCRETE:
            params[2] = float(rng.uniform(0.05, 0.6))
        topo = int(rng.integers(0, 3))
        n = int(rng.integers(20, 100))
        cfg = sp.make_config(n, int(rng.integers(1, 3)), 2, rho=float(rng.uniform(0.6, 1.6)),
                             ei=float(rng.uniform(0.3, 0.8)), gamma=float(rng.uniform(0.3, 2.0)),
                             conn=(0.1 if topo == sp.CONN_RANDOM else 4.0 / (n - 1)),
                             dt=float(rng.choice([1.0, 0.5])), topo=topo, neuron=neuron,
                             nparams=tuple(params), synapse=synapse,
                             backend=int(rng.integers(0, 2)), sparams=O.SYNAPSE_PARAMS[synapse])
        check(cfg, seed=int(rng.integers(1, 10**6)), T=40)
