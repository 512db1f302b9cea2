"""Construction on the device: the power iteration that scales the recurrent
weights gives the host's bits, so reservoirs created with it keep weight
parity with the host-only build (and so with the reference)."""
import numpy as np
import pytest

import spires_b200 as sp

pytestmark = pytest.mark.gpu

GL = (1.0, 0.0, 0.0, 20.0, 0.7, 64.0, 0.1, 2.0)


def spectral(lib, rp, col, w, dev):
    out = np.zeros(1)
    st = lib.spires_ext_spectral_radius(len(rp) - 1, rp.ctypes.data_as(sp._i64p),
                                        col.ctypes.data_as(sp._i32p), sp.dptr(w), dev,
                                        sp.dptr(out))
    assert st == sp.SPIRES_OK
    return out[0]


@pytest.mark.parametrize("n,conn,topo", [
    (3000, 0.05, sp.CONN_RANDOM),
    (4097, 12.0 / 4096, sp.CONN_SMALL_WORLD),
    (5000, 20.0 / 4999, sp.CONN_SCALE_FREE),
    (257, 0.3, sp.CONN_RANDOM),
])
def test_device_power_iteration_matches_host(n, conn, topo):
    cfg = sp.make_config(n, 1, 1, rho=1.1, conn=conn, topo=topo, neuron=sp.FLIF_GL, nparams=GL)
    m = sp.HostModel(cfg, seed=17)
    rp, col, w = m.csr()
    rp = np.ascontiguousarray(rp, np.int64)
    col = np.ascontiguousarray(col, np.int32)
    w = np.ascontiguousarray(w, np.float64)
    h = spectral(m.lib, rp, col, w, 0)
    d = spectral(m.lib, rp, col, w, 1)
    assert np.float64(h).view(np.uint64) == np.float64(d).view(np.uint64), (h, d)
    # a matrix with empty rows and a scaled copy
    w2 = w * 3.0
    w2[rp[1]:rp[n // 2]] = 0.0
    assert np.float64(spectral(m.lib, rp, col, w2, 0)).view(np.uint64) == \
        np.float64(spectral(m.lib, rp, col, w2, 1)).view(np.uint64)


def test_created_reservoir_keeps_weight_parity():
    # 2000 x 2000 at 8 %: 320k edges, above the device threshold
    cfg = sp.make_config(2000, 2, 1, rho=0.95, conn=0.08, topo=sp.CONN_RANDOM,
                         neuron=sp.FLIF_GL, nparams=GL)
    r = sp.Reservoir(cfg, seed=99)
    W = r.weights()
    r.close()
    m = sp.HostModel(cfg, seed=99)
    assert m.info.nnz >= 1 << 15
    assert np.array_equal(W.view(np.uint64), m.dense().view(np.uint64))
