"""Recurrent weights injected from a dense matrix (N(0,1) weights on an
Erdos-Renyi pattern, as the small LIF_DISCRETE workload specifies): the
stored weights are the dense ones times the power-iteration scale, and the
dynamics match the oracle driven with the same weights bit for bit."""
import numpy as np
import pytest

import spires_b200 as sp
from tests import _oracle as O

pytestmark = pytest.mark.gpu


def csr_of(D):
    n = D.shape[0]
    mask = D != 0.0
    rp = np.concatenate([[0], np.cumsum(mask.sum(axis=1))]).astype(np.int64)
    cols = np.nonzero(mask)[1].astype(np.int32)
    vals = D[mask].astype(np.float64)
    return rp, cols, vals


class Injected:
    """The pieces of a host model the oracle reads, with injected weights."""

    def __init__(self, rp, col, val, w_in, w_out):
        self._csr = (rp, col, val)
        self._w_in, self._w_out = w_in, w_out

    def csr(self):
        return self._csr

    def w_in(self):
        return self._w_in

    def w_out(self):
        return self._w_out

    def edge_tau(self):
        return None


@pytest.mark.parametrize("neuron,params,gamma", [
    (sp.LIF_DISCRETE, (0.0, 1.0, 0.9, 0.0), 0.5),
    (sp.FLIF_GL, (1.0, 0.0, 0.0, 20.0, 0.7, 64.0, 0.1, 2.0), 1.0),
])
def test_injected_dense_weights(neuron, params, gamma):
    n = 400
    cfg = sp.make_config(n, 1, 1, rho=0.9, ei=0.5, gamma=gamma, conn=0.1, neuron=neuron,
                         nparams=params)
    rng = np.random.default_rng(7)
    mask = rng.random((n, n)) < 0.1
    np.fill_diagonal(mask, False)
    D = np.where(mask, rng.standard_normal((n, n)), 0.0)
    r = sp.Reservoir(cfg, seed=5)
    r.set_weights(D, rescale=True)
    W = r.weights()
    rp, col, val = csr_of(D)
    sr = np.zeros(1)
    assert r.lib.spires_ext_spectral_radius(n, rp.ctypes.data_as(sp._i64p),
                                            col.ctypes.data_as(sp._i32p), sp.dptr(val), 0,
                                            sp.dptr(sr)) == sp.SPIRES_OK
    f = 0.9 / sr[0]
    expected = np.where(mask, f * D, 0.0)
    assert np.array_equal(W.view(np.uint64), expected.view(np.uint64))
    u = np.random.default_rng(1).uniform(-1, 1.5, (300, 1))
    phi, R, _ = r.run_record(u)
    ras = sp.unpack_raster(R, n)
    orc = O.Oracle(cfg, Injected(rp, col, f * val, r.w_in(), r.readout()))
    phi_o, ras_o, _ = orc.run(u)
    r.close()
    assert np.array_equal(ras, ras_o)
    assert np.array_equal(phi.view(np.uint64), phi_o.view(np.uint64))
