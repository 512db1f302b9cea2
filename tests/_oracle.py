"""Test-side access to the oracle (checker only; never imported by the product).

Two checkers live under oracle/:
  * oracle/_ref/libspires_ref.so -- the reference spires C sources compiled
    unchanged against the netlib-order BLAS shim (bit-parity reference);
  * oracle/build/liboracle.so   -- the C restatement in oracle/spires_oracle.c.
"""
import ctypes as C
import os
import subprocess

import spires_b200 as sp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE = os.path.join(ROOT, "oracle")
REF_SO = os.path.join(ORACLE, "_ref", "libspires_ref.so")
REF_OPENBLAS_SO = os.path.join(ORACLE, "_ref", "libspires_ref_openblas.so")
ORACLE_SO = os.path.join(ORACLE, "build", "liboracle.so")

_cache = {}


def have_ref():
    return os.path.exists(REF_SO)


def ref_lib(kind="netlib"):
    path = REF_SO if kind == "netlib" else REF_OPENBLAS_SO
    if path not in _cache:
        if not os.path.exists(path):
            subprocess.run(["make", "-C", ORACLE, "ref"], capture_output=True)
        lib = C.CDLL(path)
        sp.bind(lib, sp.SIGNATURES)
        _cache[path] = lib
    return _cache[path]


def oracle_lib():
    if ORACLE_SO not in _cache:
        if not os.path.exists(ORACLE_SO):
            subprocess.run(["make", "-C", ORACLE, "oracle"], check=True, capture_output=True)
        lib = C.CDLL(ORACLE_SO)
        _cache[ORACLE_SO] = lib
    return _cache[ORACLE_SO]


import numpy as np

_dp = C.POINTER(C.c_double)


class OrcModel(C.Structure):
    """orc_model of oracle/spires_oracle.h."""

    _fields_ = [
        ("neuron_type", C.c_int), ("synapse_type", C.c_int),
        ("n", C.c_int), ("din", C.c_int), ("dout", C.c_int),
        ("dt", C.c_double), ("input_strength", C.c_double),
        ("neuron_params", _dp), ("synapse_params", _dp),
        ("row_ptr", C.POINTER(C.c_int64)), ("col", C.POINTER(C.c_int32)), ("val", _dp),
        ("w_in", _dp), ("w_out", _dp), ("edge_tau", _dp),
        ("diffusive_seed", C.c_uint64),
    ]


def _bind_oracle(lib):
    lib.orc_create.restype = C.c_void_p
    lib.orc_create.argtypes = [C.POINTER(OrcModel)]
    lib.orc_free.argtypes = [C.c_void_p]
    lib.orc_reset.argtypes = [C.c_void_p]
    lib.orc_step.argtypes = [C.c_void_p, _dp]
    lib.orc_state_read.argtypes = [C.c_void_p, _dp, _dp]
    lib.orc_output.argtypes = [C.c_void_p, _dp]
    lib.orc_run.argtypes = [C.c_void_p, _dp, C.c_size_t, _dp, C.POINTER(C.c_uint8), _dp]
    lib.orc_train_online.argtypes = [C.c_void_p, _dp, C.c_double, _dp]
    lib.orc_train_rls.restype = C.c_int
    lib.orc_train_rls.argtypes = [C.c_void_p, _dp, _dp, C.c_size_t, C.c_double, C.c_double, _dp]
    lib.orc_ridge.restype = C.c_int
    lib.orc_ridge.argtypes = [_dp, _dp, C.c_size_t, C.c_size_t, C.c_int, C.c_int, C.c_double,
                              _dp]
    return lib


class Oracle:
    """CPU restatement driven with the weights of a built host model."""

    def __init__(self, cfg, hm, w_out=None, seed=0):
        self.lib = _bind_oracle(oracle_lib())
        self.cfg = cfg
        rp, col, val = hm.csr()
        self._keep = [rp, col, val, hm.w_in().copy(),
                      (hm.w_out() if w_out is None else w_out).copy()]
        tau = hm.edge_tau() if cfg.synapse_type == sp.SYN_PSC_HET else None
        self._keep.append(tau)
        m = OrcModel()
        m.neuron_type = cfg.neuron_type
        m.synapse_type = cfg.synapse_type
        m.n, m.din, m.dout = cfg.num_neurons, cfg.num_inputs, cfg.num_outputs
        m.dt, m.input_strength = cfg.dt, cfg.input_strength
        m.neuron_params = cfg.neuron_params
        m.synapse_params = cfg.synapse_params
        m.row_ptr = rp.ctypes.data_as(C.POINTER(C.c_int64))
        m.col = col.ctypes.data_as(C.POINTER(C.c_int32))
        m.val = sp.dptr(val)
        m.w_in = sp.dptr(self._keep[3])
        m.w_out = sp.dptr(self._keep[4])
        m.edge_tau = sp.dptr(tau) if tau is not None else None
        m.diffusive_seed = seed
        self.m = m
        self.h = self.lib.orc_create(C.byref(m))
        self.n = int(cfg.num_neurons)
        self.dout = int(cfg.num_outputs)

    def __del__(self):
        try:
            self.lib.orc_free(self.h)
        except Exception:
            pass

    def run(self, u, T=None, y=False):
        if u is not None:
            u = np.ascontiguousarray(u, dtype=np.float64)
            T = u.shape[0]
        phi = np.empty((T, self.n))
        ras = np.empty((T, self.n), np.uint8)
        Y = np.empty((T, max(self.dout, 1))) if y else None
        self.lib.orc_run(self.h, None if u is None else sp.dptr(u), T, sp.dptr(phi),
                         ras.ctypes.data_as(C.POINTER(C.c_uint8)),
                         sp.dptr(Y) if Y is not None else None)
        return phi, ras, Y

    def reset(self):
        self.lib.orc_reset(self.h)

    def step(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        self.lib.orc_step(self.h, sp.dptr(u))

    def train_online(self, target, lr, w_out):
        t = np.ascontiguousarray(target, dtype=np.float64)
        self.lib.orc_train_online(self.h, sp.dptr(t), lr, sp.dptr(w_out))

    def train_rls(self, u, y, delta, lam):
        u = np.ascontiguousarray(u, np.float64)
        y = np.ascontiguousarray(y, np.float64)
        W = np.empty((self.dout, self.n))
        assert self.lib.orc_train_rls(self.h, sp.dptr(u), sp.dptr(y), u.shape[0], delta, lam,
                                      sp.dptr(W)) == 0
        return W


def oracle_ridge(X, Y, lam, washout=0):
    lib = _bind_oracle(oracle_lib())
    X = np.ascontiguousarray(X, np.float64)
    Y = np.ascontiguousarray(Y, np.float64)
    T, n = X.shape
    dout = Y.shape[1]
    W = np.empty((dout, n))
    rc = lib.orc_ridge(sp.dptr(X), sp.dptr(Y), T, washout, n, dout, lam, sp.dptr(W))
    assert rc == 0
    return W


def ref_trajectory(cfg, seed, u, lib=None):
    """States and spikes of the compiled reference after every spires_step."""
    r = sp.Reservoir(cfg, lib=lib or ref_lib(), seed=seed)
    T = u.shape[0]
    phi = np.empty((T, r.n))
    ras = np.empty((T, r.n), np.uint8)
    for t in range(T):
        r.step(u[t])
        phi[t] = r.state()
        ras[t] = r.spikes() != 0.0
    r.close()
    return phi, ras


# Parameter sets used by the parity tests (neuron_params layouts of spires.h).
NEURON_PARAMS = {
    sp.LIF_DISCRETE: (0.0, 1.0, 0.3, 0.05),
    sp.LIF_BIO: (0.0, 1.0, 5.0, 0.85),
    sp.FLIF_CAPUTO: (1.0, 0.2, 0.0, 1.0, 0.0, 1.5, 0.7, 2.0, 40.0),
    sp.FLIF_GL: (1.0, 0.0, 0.0, 20.0, 0.7, 64.0, 0.1, 2.0),
    sp.FLIF_DIFFUSIVE: (1.0, 0.0, 0.0, 5.0, 1.0, 3.0, 0.85),
}
SYNAPSE_PARAMS = {
    sp.SYN_SIMPLE: None,
    sp.SYN_PSC_HOM: (3.0,),
    sp.SYN_PSC_HET: (1.0, 10.0),
    sp.SYN_FRAC: (0.6, 4.0, 20.0),
    sp.SYN_FRAC_MEXP: (0.5, 4.0, 1.0, 40.0, 5),
}
