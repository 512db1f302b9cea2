"""Host construction parity: W, W_in, W_out drawn with rand() exactly as the
reference draws them (src/reservoir.c:308-571). Runs on the CPU only: the
library's host-only model build is compared with the reference compiled from
source (oracle/_ref)."""
import numpy as np
import pytest

import spires_b200 as sp
from tests import _oracle

pytestmark = pytest.mark.skipif(not _oracle.have_ref(), reason="reference build absent")

GL = (1.0, 0.0, 0.0, 20.0, 0.7, 64.0, 0.1, 2.0)

CASES = [
    # n, topo, conn, din, dout, neuron, params, synapse, backend, sparams
    (60, sp.CONN_RANDOM, 0.1, 1, 1, sp.LIF_DISCRETE, (0, 1, 0.9, 0), sp.SYN_SIMPLE, 0, None),
    (200, sp.CONN_RANDOM, 0.05, 3, 2, sp.FLIF_GL, GL, sp.SYN_SIMPLE, 0, None),
    (200, sp.CONN_SMALL_WORLD, 10 / 199, 1, 1, sp.FLIF_GL, GL, sp.SYN_SIMPLE, 0, None),
    (300, sp.CONN_SMALL_WORLD, 0.2, 2, 1, sp.FLIF_GL, GL, sp.SYN_SIMPLE, 1, None),
    (3, sp.CONN_SMALL_WORLD, 0.9, 1, 1, sp.LIF_BIO, (0, 1, 20, 0.1), sp.SYN_SIMPLE, 0, None),
    (250, sp.CONN_SCALE_FREE, 5 / 249, 13, 10, sp.FLIF_GL, GL, sp.SYN_SIMPLE, 0, None),
    (150, sp.CONN_SCALE_FREE, 0.1, 1, 1, sp.LIF_DISCRETE, (0, 1, 0.9, 0), sp.SYN_SIMPLE, 1, None),
    (2, sp.CONN_SCALE_FREE, 0.5, 1, 1, sp.LIF_DISCRETE, (0, 1, 0.9, 0), sp.SYN_SIMPLE, 0, None),
    (1000, sp.CONN_SCALE_FREE, 0.1, 1, 1, sp.LIF_DISCRETE, (0, 1, 0.9, 0), sp.SYN_SIMPLE, 0, None),
    (600, sp.CONN_RANDOM, 0.3, 1, 1, sp.LIF_DISCRETE, (0, 1, 0.9, 0), sp.SYN_SIMPLE, 0, None),
    (120, sp.CONN_RANDOM, 0.1, 1, 1, sp.FLIF_GL, GL, sp.SYN_PSC_HET, 0, (1.0, 20.0)),
    (80, sp.CONN_SMALL_WORLD, 0.1, 1, 1, sp.FLIF_GL, GL, sp.SYN_PSC_HET, 1, (2.0, 8.0)),
    (100, sp.CONN_SCALE_FREE, 0.03, 1, 1, sp.FLIF_GL, GL, sp.SYN_FRAC_MEXP, 0,
     (0.5, 5.0, 1.0, 50.0, 6)),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"n{c[0]}-topo{c[1]}-syn{c[7]}-be{c[8]}")
@pytest.mark.parametrize("seed", [1, 42])
def test_weights_match_reference(case, seed):
    n, topo, conn, din, dout, neuron, params, syn, be, sparams = case
    cfg = sp.make_config(n, din, dout, rho=0.93, ei=0.6, gamma=0.5, conn=conn, dt=1.0,
                         topo=topo, neuron=neuron, nparams=params, synapse=syn, backend=be,
                         sparams=sparams)
    mine = sp.HostModel(cfg, seed=seed)
    ref = sp.Reservoir(cfg, lib=_oracle.ref_lib(), seed=seed)
    Wr = ref.weights()
    Wm = mine.dense()
    assert np.array_equal(Wr.view(np.uint64), Wm.view(np.uint64)) or np.array_equal(Wr, Wm)
    assert np.array_equal(ref.readout(), mine.w_out())
    # W_in comes first in the draw order: replay it with the C library's rand()
    sp.libc.srand(seed)
    RAND_MAX = 2147483647.0
    win = np.empty(n * din)
    for k in range(n * din):
        mag = sp.libc.rand() / RAND_MAX
        win[k] = mag if sp.libc.rand() / RAND_MAX < 0.6 else -mag
    assert np.array_equal(win.reshape(n, din), mine.w_in())
    ref.close()


def test_rand_stream_position_after_create():
    """The next rand() after construction is the same in both libraries, so
    callers that build several reservoirs from one seed get the same sequence."""
    cfg = sp.make_config(300, 2, 2, conn=5 / 299, topo=sp.CONN_SCALE_FREE, neuron=sp.FLIF_GL,
                         nparams=GL)
    sp.HostModel(cfg, seed=7)
    a = [sp.libc.rand() for _ in range(4)]
    r = sp.Reservoir(cfg, lib=_oracle.ref_lib(), seed=7)
    b = [sp.libc.rand() for _ in range(4)]
    r.close()
    assert a == b


def test_invalid_configs_rejected():
    lib = sp.load()
    import ctypes as C
    h = C.c_void_p()
    for kw in [dict(dt=0.0), dict(dt=0.3), dict(dt=1.5), dict(neuron=9), dict(synapse=9)]:
        cfg = sp.make_config(10, **kw)
        assert lib.spires_ext_model_build(C.byref(cfg), C.byref(h)) == sp.SPIRES_ERR_INVALID_ARG
    assert lib.spires_reservoir_create(None, C.byref(h)) == sp.SPIRES_ERR_INVALID_ARG


# ---- private generator with the srand/rand sequence (parallel batch builds)
@pytest.mark.parametrize("seed", [0, 1, 42, 2**31 - 1, 2**31 + 5, 2**32 - 1])
@pytest.mark.parametrize("topo", [sp.CONN_RANDOM, sp.CONN_SMALL_WORLD, sp.CONN_SCALE_FREE])
def test_private_generator_matches_global_rand(seed, topo):
    cfg = sp.make_config(150, 2, 3, rho=1.1, ei=0.6, conn=0.07, topo=topo, neuron=sp.FLIF_GL,
                         nparams=(1.0, 0.0, 0.0, 20.0, 0.7, 32.0, 0.1, 2.0))
    a = sp.HostModel(cfg, seed=seed)
    b = sp.HostModel(cfg, seed=seed, private=True)
    for x, y in zip(a.csr(), b.csr()):
        assert np.array_equal(x, y)
    assert np.array_equal(a.w_in(), b.w_in())
    assert np.array_equal(a.w_out(), b.w_out())


@pytest.mark.parametrize("n,conn", [(1500, 0.3), (1500, 0.0005), (2500, 0.02)])
@pytest.mark.parametrize("topo", [sp.CONN_RANDOM, sp.CONN_SMALL_WORLD, sp.CONN_SCALE_FREE])
def test_private_generator_matches_global_rand_large(n, conn, topo):
    """Dense and near-empty graphs (edge runs that cross rows and draw blocks),
    an uneven sign ratio, and per-edge synapse draws after the topology."""
    cfg = sp.make_config(n, 1, 2, rho=0.9, ei=0.37, conn=conn, topo=topo, neuron=sp.FLIF_GL,
                         nparams=(1.0, 0.0, 0.0, 20.0, 0.7, 32.0, 0.1, 2.0),
                         synapse=sp.SYN_PSC_HET, sparams=(1.0, 20.0))
    a = sp.HostModel(cfg, seed=11)
    b = sp.HostModel(cfg, seed=11, private=True)
    for x, y in zip(a.csr(), b.csr()):
        assert np.array_equal(x, y)
    assert np.array_equal(a.w_in(), b.w_in())
    assert np.array_equal(a.w_out(), b.w_out())


def test_private_generator_leaves_global_rand_alone():
    sp.libc.srand(7)
    first = sp.libc.rand()
    sp.libc.srand(7)
    cfg = sp.make_config(64, 1, 1, conn=0.1)
    sp.HostModel(cfg, seed=99, private=True)
    assert sp.libc.rand() == first


@pytest.mark.parametrize("topo", [sp.CONN_SMALL_WORLD, sp.CONN_SCALE_FREE])
def test_out_of_range_connectivity_truncates_as_x86(topo):
    """A degree parameter (connectivity * (n - 1) + 0.5) that is NaN or beyond
    the int range converts to INT_MIN, as the reference's cast does on
    x86-64, and so falls to the smallest degree -- the same graph as
    connectivity 0."""
    base = sp.HostModel(sp.make_config(200, conn=0.0, topo=topo), seed=5, private=True).csr()
    for c in (1e12, -1e12, float("nan")):
        g = sp.HostModel(sp.make_config(200, conn=c, topo=topo), seed=5, private=True).csr()
        for x, y in zip(base, g):
            assert np.array_equal(x, y)


def test_out_of_range_ring_length_rejected():
    lib = sp.load()
    import ctypes as C
    h = C.c_void_p()
    # beyond the int range: INT_MIN, rejected as a ring length below one
    cfg = sp.make_config(10, neuron=sp.FLIF_GL, nparams=(1.0, 0.0, 0.0, 20.0, 0.7, 1e300, 0.1, 2.0))
    assert lib.spires_ext_model_build(C.byref(cfg), C.byref(h)) == sp.SPIRES_ERR_INVALID_ARG
    # NaN fails T_mem > 0 and takes the default ring, as in the reference
    cfg = sp.make_config(10, neuron=sp.FLIF_GL,
                         nparams=(1.0, 0.0, 0.0, 20.0, 0.7, float("nan"), 0.1, 2.0))
    m = sp.HostModel(cfg, seed=1)
    assert m.n == 10


def test_model_info_reports_construction_times():
    cfg = sp.make_config(1500, conn=0.05, topo=sp.CONN_SCALE_FREE)
    m = sp.HostModel(cfg, seed=3, private=True)
    assert m.info.topology_ms > 0.0
    assert m.info.spectral_ms > 0.0
    assert m.info.nnz > 0


@pytest.mark.skipif(not _oracle.have_ref(), reason="reference build absent")
@pytest.mark.parametrize("topo,backend,syn", [(5, 0, sp.SYN_SIMPLE), (sp.CONN_RANDOM, 7, sp.SYN_SIMPLE),
                                              (sp.CONN_SMALL_WORLD, 3, sp.SYN_PSC_HET)])
def test_unlisted_topology_and_backend_values_as_the_reference(topo, backend, syn):
    """The reference accepts any topology value (no recurrent edges for one it
    does not list) and stores dense for any backend but SPARSE; same weights
    and the same draw count here."""
    sparams = (1.0, 20.0) if syn == sp.SYN_PSC_HET else None
    cfg = sp.make_config(90, 2, 2, rho=0.9, ei=0.6, conn=0.1, topo=topo, neuron=sp.FLIF_GL,
                         nparams=GL, synapse=syn, backend=backend, sparams=sparams)
    mine = sp.HostModel(cfg, seed=4)
    ref = sp.Reservoir(cfg, lib=_oracle.ref_lib(), seed=4)
    assert np.array_equal(ref.weights(), mine.dense())
    assert np.array_equal(ref.readout(), mine.w_out())
    ref.close()
    if topo == 5:
        assert mine.info.nnz == 0


@pytest.mark.skipif(not _oracle.have_ref(), reason="reference build absent")
def test_randomised_configurations_match_reference():
    """Randomised sizes, densities, sign ratios (including beyond [0, 1]),
    spectral radii, topologies, synapse types and backends: the same W, W_out
    and draw count as the reference's create."""
    rng = np.random.default_rng(2025)
    syn_params = {sp.SYN_SIMPLE: None, sp.SYN_PSC_HOM: (3.0,), sp.SYN_PSC_HET: (1.0, 20.0),
                  sp.SYN_FRAC: (0.6, 2.0, 8.0), sp.SYN_FRAC_MEXP: (0.5, 5.0, 1.0, 50.0, 4)}
    for trial in range(30):
        n = int(rng.integers(2, 120))
        syn = int(rng.integers(0, 5))
        cfg = sp.make_config(n, int(rng.integers(1, 4)), int(rng.integers(1, 4)),
                             rho=float(rng.choice([0.0, 0.5, 1.3, -0.7])),
                             ei=float(rng.choice([0.0, 0.25, 0.5, 1.0, 1.5, -0.2])),
                             gamma=0.5, conn=float(rng.choice([0.0, 0.01, 0.1, 0.5, 1.0, 2.0])),
                             topo=int(rng.integers(0, 3)), neuron=sp.FLIF_GL, nparams=GL,
                             synapse=syn, backend=int(rng.integers(0, 2)),
                             sparams=syn_params[syn])
        seed = int(rng.integers(1, 2**31 - 1))
        mine = sp.HostModel(cfg, seed=seed)
        after_mine = sp.libc.rand()
        ref = sp.Reservoir(cfg, lib=_oracle.ref_lib(), seed=seed)
        after_ref = sp.libc.rand()
        Wr = ref.weights()
        Wo = ref.readout()
        ref.close()
        assert np.array_equal(Wr, mine.dense()), trial
        assert np.array_equal(Wo, mine.w_out()), trial
        assert after_mine == after_ref, trial  # the same number of draws
