"""State checkpoint (spires_ext_state_bytes / _save / _load): a reservoir
saved mid-run and loaded back -- into itself, or into a fresh reservoir built
from the same configuration and seed -- continues bit for bit as the
uninterrupted run does, for every neuron model and every synapse model; the
checkpoint carries the readout; a buffer of another size is refused."""
import ctypes as C

import numpy as np
import pytest

import spires_b200 as sp
from tests import _oracle as O

pytestmark = pytest.mark.gpu

# every neuron model and every synapse model at least once
CASES = [
    (sp.LIF_DISCRETE, sp.SYN_SIMPLE),
    (sp.LIF_BIO, sp.SYN_PSC_HOM),
    (sp.FLIF_CAPUTO, sp.SYN_PSC_HET),
    (sp.FLIF_GL, sp.SYN_FRAC),
    (sp.FLIF_DIFFUSIVE, sp.SYN_FRAC_MEXP),
    (sp.FLIF_GL, sp.SYN_SIMPLE),
]


def cfg_for(neuron, synapse, n=150):
    return sp.make_config(n, 2, 2, rho=1.2, ei=0.55, gamma=1.2, conn=0.06, neuron=neuron,
                          nparams=O.NEURON_PARAMS[neuron], synapse=synapse,
                          sparams=O.SYNAPSE_PARAMS[synapse])


def save(r):
    nb = r.lib.spires_ext_state_bytes(r.h)
    assert nb > 0
    buf = (C.c_char * nb)()
    assert r.lib.spires_ext_state_save(r.h, buf, nb) == sp.SPIRES_OK
    return buf


def load(r, buf, nb=None):
    return r.lib.spires_ext_state_load(r.h, buf, len(buf) if nb is None else nb)


@pytest.mark.parametrize("neuron,synapse", CASES)
def test_checkpoint_resumes_bit_for_bit(neuron, synapse):
    cfg = cfg_for(neuron, synapse)
    u = np.random.default_rng(1).uniform(-1.0, 1.5, (160, 2))
    a = sp.Reservoir(cfg, seed=31)
    a.run_record(u[:70])
    buf = save(a)
    p1, r1, _ = a.run_record(u[70:])  # the uninterrupted continuation
    assert load(a, buf) == sp.SPIRES_OK
    p2, r2, _ = a.run_record(u[70:])  # the same steps again from the loaded state
    a.close()
    b = sp.Reservoir(cfg, seed=31)  # a fresh reservoir resumed from the checkpoint
    assert load(b, buf) == sp.SPIRES_OK
    p3, r3, _ = b.run_record(u[70:])
    b.close()
    for p, r in ((p2, r2), (p3, r3)):
        assert np.array_equal(r, r1)
        assert np.array_equal(p.view(np.uint64), p1.view(np.uint64))


def test_checkpoint_carries_the_readout():
    cfg = cfg_for(sp.FLIF_GL, sp.SYN_SIMPLE)
    rng = np.random.default_rng(2)
    u = rng.uniform(-1.0, 1.5, (200, 2))
    y = rng.standard_normal((200, 2))
    r = sp.Reservoir(cfg, seed=5)
    W0 = r.readout()
    buf = save(r)
    r.train_ridge(u, y, 1e-3)
    assert not np.array_equal(r.readout(), W0)
    assert load(r, buf) == sp.SPIRES_OK
    assert np.array_equal(r.readout(), W0)
    # the device copy is the restored one too: the readout of the state
    r.run(u[:10])
    out = r.output()
    v = r.state()
    scale = float((np.abs(W0) @ np.abs(v)).max())
    assert np.max(np.abs(out - W0 @ v)) <= 1e-12 * max(scale, 1e-300)
    r.close()


def test_checkpoint_of_another_size_is_refused():
    a = sp.Reservoir(cfg_for(sp.FLIF_GL, sp.SYN_SIMPLE), seed=3)
    buf = save(a)
    a.close()
    b = sp.Reservoir(cfg_for(sp.FLIF_GL, sp.SYN_SIMPLE, n=151), seed=3)
    assert load(b, buf) == sp.SPIRES_ERR_INVALID_ARG
    b.close()


def test_checkpoint_of_fewer_outputs_is_refused():
    """Same neurons and models, another readout width: the checkpoint is
    smaller than this reservoir's, so it is refused before any byte past its
    end could be read."""
    def cfg(dout):
        return sp.make_config(150, 2, dout, rho=1.2, ei=0.55, gamma=1.2, conn=0.06,
                              neuron=sp.FLIF_GL, nparams=O.NEURON_PARAMS[sp.FLIF_GL])
    a = sp.Reservoir(cfg(2), seed=3)
    buf = save(a)
    a.close()
    b = sp.Reservoir(cfg(3), seed=3)
    before = b.readout().copy()
    assert load(b, buf) == sp.SPIRES_ERR_INVALID_ARG
    # even when the caller claims the size this reservoir expects
    assert load(b, buf, b.lib.spires_ext_state_bytes(b.h)) == sp.SPIRES_ERR_INVALID_ARG
    assert np.array_equal(b.readout(), before)
    b.close()


def test_checkpoint_of_other_dynamics_is_refused():
    """Same sizes, but another seed (another graph) or another parameter set:
    the header's hash differs and the load is refused with the state kept."""
    cfg = cfg_for(sp.FLIF_GL, sp.SYN_SIMPLE)
    u = np.random.default_rng(4).uniform(-1.0, 1.5, (40, 2))
    a = sp.Reservoir(cfg, seed=3)
    a.run_record(u)
    buf = save(a)
    a.close()
    b = sp.Reservoir(cfg, seed=4)
    b.run_record(u[:5])
    v0 = b.state().copy()
    assert load(b, buf) == sp.SPIRES_ERR_INVALID_ARG
    assert np.array_equal(b.state(), v0)
    b.close()
    params = list(O.NEURON_PARAMS[sp.FLIF_GL])
    params[6] += 0.25  # bias
    cfg2 = sp.make_config(150, 2, 2, rho=1.2, ei=0.55, gamma=1.2, conn=0.06,
                          neuron=sp.FLIF_GL, nparams=tuple(params))
    c = sp.Reservoir(cfg2, seed=3)
    assert load(c, buf) == sp.SPIRES_ERR_INVALID_ARG
    c.close()


def test_checkpoint_buffer_lengths():
    r = sp.Reservoir(cfg_for(sp.LIF_DISCRETE, sp.SYN_SIMPLE), seed=9)
    nb = r.lib.spires_ext_state_bytes(r.h)
    small = (C.c_char * (nb - 1))()
    assert r.lib.spires_ext_state_save(r.h, small, nb - 1) == sp.SPIRES_ERR_INVALID_ARG
    buf = save(r)
    assert load(r, buf, nb - 1) == sp.SPIRES_ERR_INVALID_ARG
    assert load(r, buf, nb + 1) == sp.SPIRES_ERR_INVALID_ARG
    assert load(r, buf) == sp.SPIRES_OK
    r.close()
