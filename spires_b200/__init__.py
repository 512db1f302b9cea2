"""spires_b200 -- B200-native drop-in for the spires reservoir C API.

The product is the C-ABI shared library ``spires_b200/lib/libspires.so``
(``include/spires.h`` + ``include/spires_ext.h``). This module only loads it
with ctypes and offers thin Python wrappers used by the tests, the benchmark
and ``__graft_entry__``. There is no Python or CPU fallback: if the library is
missing, :func:`load` raises.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libspires.so")

# enums of include/spires.h
SPIRES_OK, SPIRES_ERR_INVALID_ARG, SPIRES_ERR_ALLOC, SPIRES_ERR_INTERNAL = range(4)
CONN_RANDOM, CONN_SMALL_WORLD, CONN_SCALE_FREE = range(3)
LIF_DISCRETE, LIF_BIO, FLIF_CAPUTO, FLIF_GL, FLIF_DIFFUSIVE = range(5)
SYN_SIMPLE, SYN_PSC_HOM, SYN_PSC_HET, SYN_FRAC, SYN_FRAC_MEXP = range(5)
BACKEND_SPARSE, BACKEND_DENSE = range(2)

_dp = C.POINTER(C.c_double)
_u32p = C.POINTER(C.c_uint32)
_i64p = C.POINTER(C.c_int64)
_fp = C.POINTER(C.c_float)
_i32p = C.POINTER(C.c_int32)


class Config(C.Structure):
    """spires_reservoir_config (include/spires.h)."""

    _fields_ = [
        ("num_neurons", C.c_size_t),
        ("num_inputs", C.c_size_t),
        ("num_outputs", C.c_size_t),
        ("spectral_radius", C.c_double),
        ("ei_ratio", C.c_double),
        ("input_strength", C.c_double),
        ("connectivity", C.c_double),
        ("dt", C.c_double),
        ("connectivity_type", C.c_int),
        ("neuron_type", C.c_int),
        ("neuron_params", _dp),
        ("synapse_type", C.c_int),
        ("synapse_backend", C.c_int),
        ("synapse_params", _dp),
    ]


class OptBudget(C.Structure):
    _fields_ = [("data_fraction", C.c_double), ("num_seeds", C.c_int),
                ("time_limit_sec", C.c_double), ("_reserved_i0", C.c_int),
                ("_reserved_d0", C.c_double)]


class OptScore(C.Structure):
    _fields_ = [("lambda_var", C.c_double), ("lambda_cost", C.c_double),
                ("metric", C.c_int), ("_reserved_i0", C.c_int)]


class OptResult(C.Structure):
    _fields_ = [("best_config", Config), ("best_log10_ridge", C.c_double),
                ("best_score", C.c_double), ("metric_mean", C.c_double),
                ("metric_std", C.c_double)]


class ModelInfo(C.Structure):
    _fields_ = [("num_neurons", C.c_size_t), ("num_inputs", C.c_size_t),
                ("num_outputs", C.c_size_t), ("nnz", C.c_size_t), ("ring_len", C.c_int),
                ("micro_steps", C.c_int), ("syn_ring_len", C.c_int),
                ("syn_components", C.c_int),
                ("spectral_radius_before_rescale", C.c_double), ("topology_ms", C.c_double),
                ("spectral_ms", C.c_double)]


class Launch(C.Structure):
    _fields_ = [("ctas", C.c_int), ("warps_max", C.c_int), ("variant", C.c_int),
                ("stages", C.c_int), ("rows", C.c_int), ("csr_global", C.c_int),
                ("l2_pin", C.c_int)]


class RidgeOpts(C.Structure):
    _fields_ = [("gram_mode", C.c_int), ("max_refine", C.c_int), ("refine_tol", C.c_double),
                ("washout", C.c_size_t), ("gram_slices", C.c_int)]


class RidgeReport(C.Structure):
    _fields_ = [("gram_mode_used", C.c_int), ("refine_iters", C.c_int),
                ("rel_residual", C.c_double), ("collect_ms", C.c_double),
                ("gram_ms", C.c_double), ("factor_ms", C.c_double),
                ("refine_ms", C.c_double), ("factor_failed", C.c_int),
                ("lu_fallback", C.c_int), ("dual", C.c_int), ("solve_ms", C.c_double)]


class AgileOpts(C.Structure):
    _fields_ = [("mu", C.c_double), ("eta_min", C.c_double), ("eta_max", C.c_double),
                ("patience0", C.c_double), ("patience_decay", C.c_double),
                ("refine_step", C.c_double), ("refine_max_iters", C.c_int),
                ("refine_no_improve", C.c_int), ("spsa_eps", C.c_double),
                ("reflect_at_bounds", C.c_int), ("seed", C.c_uint64), ("verbose", C.c_int)]


class AgileReport(C.Structure):
    _fields_ = [("best_loss", C.c_double), ("best_iter", C.c_int), ("total_evals", C.c_int),
                ("total_iters", C.c_int), ("exited_refinement", C.c_int)]


LOSS_FN = C.CFUNCTYPE(C.c_double, C.POINTER(C.c_double), C.c_int, C.c_void_p)

# Public symbols of include/spires.h and include/spires_ext.h with their
# ctypes signatures (restype, argtypes).
_VP = C.c_void_p
SIGNATURES = {
    "spires_reservoir_create": (C.c_int, [C.POINTER(Config), C.POINTER(_VP)]),
    "spires_reservoir_destroy": (None, [_VP]),
    "spires_reservoir_reset": (C.c_int, [_VP]),
    "spires_step": (C.c_int, [_VP, _dp]),
    "spires_run": (_dp, [_VP, _dp, C.c_size_t]),
    "spires_train_online": (C.c_int, [_VP, _dp, C.c_double]),
    "spires_train_ridge": (C.c_int, [_VP, _dp, _dp, C.c_size_t, C.c_double]),
    "spires_train_rls": (C.c_int, [_VP, _dp, _dp, C.c_size_t, C.c_double, C.c_double]),
    "spires_coarse_grain": (C.c_int, [_VP, C.c_double, C.POINTER(_VP)]),
    "spires_copy_reservoir_state": (_dp, [_VP]),
    "spires_read_reservoir_state": (C.c_int, [_VP, _dp]),
    "spires_read_spike_state": (C.c_int, [_VP, _dp]),
    "spires_copy_weights": (_dp, [_VP]),
    "spires_read_weights": (C.c_int, [_VP, _dp]),
    "spires_compute_output": (C.c_int, [_VP, _dp]),
    "spires_copy_readout": (_dp, [_VP]),
    "spires_read_readout": (C.c_int, [_VP, _dp]),
    "spires_num_neurons": (C.c_size_t, [_VP]),
    "spires_num_inputs": (C.c_size_t, [_VP]),
    "spires_num_outputs": (C.c_size_t, [_VP]),
    "spires_optimize": (C.c_int, [C.POINTER(Config), C.POINTER(OptBudget), C.c_int,
                                  C.POINTER(OptScore), C.POINTER(OptResult), _dp, _dp,
                                  C.c_size_t]),
}
EXT_SIGNATURES = {
    "spires_ext_model_build": (C.c_int, [C.POINTER(Config), C.POINTER(_VP)]),
    "spires_ext_model_build_seeded": (C.c_int, [C.POINTER(Config), C.c_uint, C.POINTER(_VP)]),
    "spires_ext_model_free": (None, [_VP]),
    "spires_ext_model_info_get": (C.c_int, [_VP, C.POINTER(ModelInfo)]),
    "spires_ext_model_csr": (C.c_int, [_VP, _i64p, _i32p, _dp]),
    "spires_ext_model_w_in": (C.c_int, [_VP, _dp]),
    "spires_ext_model_w_out": (C.c_int, [_VP, _dp]),
    "spires_ext_model_edge_tau": (C.c_int, [_VP, _dp]),
    "spires_ext_model_coef": (C.c_int, [_VP, _dp]),
    "spires_ext_run_record": (C.c_int, [_VP, _dp, C.c_size_t, _dp, _u32p, _dp]),
    "spires_ext_run_device": (C.c_int, [_VP, _VP, C.c_size_t, _VP, _VP, _VP]),
    "spires_ext_sync": (C.c_int, [_VP]),
    "spires_ext_stream": (_VP, [_VP]),
    "spires_ext_spike_words": (C.c_size_t, [_VP]),
    "spires_ext_kernel_launches": (C.c_longlong, [_VP]),
    "spires_ext_read_w_in": (C.c_int, [_VP, _dp]),
    "spires_ext_get_launch": (C.c_int, [_VP, C.POINTER(Launch)]),
    "spires_ext_l2_pin_rows": (C.c_int, [_VP]),
    "spires_ext_set_launch": (C.c_int, [_VP, C.POINTER(Launch)]),
    "spires_ext_autotune": (C.c_int, [_VP, C.c_size_t]),
    "spires_ext_set_seed": (C.c_int, [_VP, C.c_uint64]),
    "spires_ext_batch_autotune": (C.c_int, [_VP, _VP, _VP, C.POINTER(C.c_int),
                                            C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "spires_ext_gram_device": (C.c_int, [_VP, C.c_size_t, C.c_size_t, C.c_size_t, C.c_int,
                                         C.c_int, _VP, _VP]),
    "spires_ext_set_wait_limit": (C.c_int, [_VP, C.c_double]),
    "spires_ext_last_device_error": (C.c_int, [_VP, C.POINTER(C.c_int),
                                              C.POINTER(C.c_longlong)]),
    "spires_ext_test_withhold_arrival": (C.c_int, [_VP, C.c_int, C.c_longlong]),
    "spires_ext_test_fail_device_alloc": (None, [C.c_longlong]),
    "spires_ext_test_live_device_allocs": (C.c_longlong, []),
    "spires_ext_state_bytes": (C.c_size_t, [_VP]),
    "spires_ext_state_save": (C.c_int, [_VP, _VP, C.c_size_t]),
    "spires_ext_state_load": (C.c_int, [_VP, _VP, C.c_size_t]),
    "spires_ext_train_ridge": (C.c_int, [_VP, _dp, _dp, C.c_size_t, C.c_double,
                                         C.POINTER(RidgeOpts), C.POINTER(RidgeReport)]),
    "spires_ext_ridge_fit": (C.c_int, [_dp, C.c_size_t, C.c_size_t, _dp, C.c_size_t, C.c_double,
                                       C.POINTER(RidgeOpts), _dp, C.POINTER(RidgeReport)]),
    "spires_ext_agile_minimize": (C.c_int, [_dp, _dp, _dp, C.c_int, LOSS_FN, _VP,
                                            C.POINTER(AgileOpts), _dp, C.POINTER(AgileReport)]),
    "spires_ext_ridge_solve_noalloc": (C.c_int, [_VP, _VP, C.c_size_t, C.c_size_t, C.c_size_t,
                                                 C.c_size_t, C.c_double, _VP, _VP]),
    "spires_ext_set_weights": (C.c_int, [_VP, _dp, C.c_int]),
    "spires_ext_spectral_radius": (C.c_int, [C.c_size_t, _i64p, _i32p, _dp, C.c_int, _dp]),
    "spires_ext_agile_batch_create": (C.c_int, [C.c_int, C.c_int, _dp, _dp, _dp,
                                                C.POINTER(AgileOpts), C.POINTER(C.c_uint64),
                                                C.POINTER(_VP)]),
    "spires_ext_agile_batch_destroy": (None, [_VP]),
    "spires_ext_agile_batch_ask": (C.c_int, [_VP, _dp, C.POINTER(C.c_int)]),
    "spires_ext_agile_batch_tell": (C.c_int, [_VP, _dp]),
    "spires_ext_agile_batch_best": (C.c_int, [_VP, C.c_int, _dp, C.POINTER(AgileReport)]),
    "spires_ext_mlp_num_params": (C.c_size_t, []),
    "spires_ext_mlp_create": (C.c_int, [C.c_uint64, C.POINTER(_VP)]),
    "spires_ext_mlp_destroy": (None, [_VP]),
    "spires_ext_mlp_get_params": (C.c_int, [_VP, _fp]),
    "spires_ext_mlp_set_params": (C.c_int, [_VP, _fp]),
    "spires_ext_mlp_loss_grad": (C.c_int, [_VP, _fp, _fp, C.c_size_t, _fp, _fp]),
    "spires_ext_mlp_train": (C.c_int, [_VP, _fp, _fp, C.c_size_t, C.c_int, C.c_int, C.c_float,
                                       C.c_uint64, _fp]),
    "spires_ext_mlp_predict": (C.c_int, [_VP, _fp, C.c_size_t, C.c_int, _fp, _fp]),
    "spires_ext_mlp_kernel_launches": (C.c_longlong, [_VP]),
    "spires_ext_batch_create": (C.c_int, [C.POINTER(Config), C.POINTER(C.c_uint), C.c_size_t,
                                          C.POINTER(_VP)]),
    "spires_ext_batch_destroy": (None, [_VP]),
    "spires_ext_batch_run": (C.c_int, [_VP, C.POINTER(_dp), C.POINTER(C.c_size_t),
                                       C.POINTER(_u32p), C.POINTER(_dp), _dp]),
    "spires_ext_batch_train_ridge": (C.c_int, [_VP, C.POINTER(_dp), C.POINTER(_dp),
                                               C.POINTER(C.c_size_t), _dp,
                                               C.POINTER(RidgeOpts), C.POINTER(_dp), _dp]),
    "spires_ext_batch_predict": (C.c_int, [_VP, C.POINTER(_dp), C.POINTER(C.c_size_t),
                                           C.POINTER(_dp), _dp]),
    "spires_ext_batch_fit_predict": (C.c_int, [_VP, C.POINTER(_dp), C.POINTER(_dp),
                                               C.POINTER(C.c_size_t), C.POINTER(C.c_size_t), _dp,
                                               C.POINTER(RidgeOpts), C.POINTER(_dp),
                                               C.POINTER(_dp), _dp]),
    "spires_ext_batch_timing": (C.c_int, [_VP, _dp, _dp]),
    "spires_ext_batch_info": (C.c_int, [_VP, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                        C.POINTER(C.c_int)]),
}

_lib = None


def build(verbose: bool = False) -> None:
    """Compile libspires.so in-tree (nvcc for sm_100a + gcc)."""
    out = subprocess.run(["make", "-C", HERE, "-j8"], capture_output=True, text=True)
    if verbose or out.returncode:
        print(out.stdout[-4000:], out.stderr[-4000:])
    if out.returncode:
        raise RuntimeError("libspires build failed")


def bind(lib: C.CDLL, table: dict) -> None:
    for name, (res, args) in table.items():
        if hasattr(lib, name):
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args


def load() -> C.CDLL:
    """Load the in-tree libspires.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} missing: run spires_b200.build() first")
        lib = C.CDLL(LIB_PATH)
        bind(lib, SIGNATURES)
        bind(lib, EXT_SIGNATURES)
        _lib = lib
    return _lib


libc = C.CDLL("libc.so.6")
libc.free.argtypes = [C.c_void_p]


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def make_config(n, din=1, dout=1, rho=0.9, ei=0.5, gamma=0.5, conn=0.1, dt=1.0,
                topo=CONN_RANDOM, neuron=LIF_DISCRETE, nparams=(0.0, 1.0, 0.9, 0.0),
                synapse=SYN_SIMPLE, backend=BACKEND_SPARSE, sparams=None):
    """Build a Config; the parameter arrays are kept alive on the returned object."""
    npar = np.ascontiguousarray(np.asarray(nparams, dtype=np.float64))
    spar = None if sparams is None else np.ascontiguousarray(np.asarray(sparams, np.float64))
    cfg = Config(n, din, dout, rho, ei, gamma, conn, dt, topo, neuron, dptr(npar), synapse,
                 backend, dptr(spar) if spar is not None else None)
    cfg._keep = (npar, spar)
    return cfg


class Reservoir:
    """Owning wrapper of a spires_reservoir handle from any spires-ABI library."""

    def __init__(self, cfg: Config, lib: C.CDLL | None = None, seed: int | None = None):
        self.lib = lib or load()
        self.cfg = cfg
        if seed is not None:
            libc.srand(seed)
        h = C.c_void_p()
        st = self.lib.spires_reservoir_create(C.byref(cfg), C.byref(h))
        if st != SPIRES_OK:
            raise RuntimeError(f"spires_reservoir_create failed: {st}")
        self.h = h
        self.n = int(cfg.num_neurons)
        self.din = int(cfg.num_inputs)
        self.dout = int(cfg.num_outputs)

    def close(self):
        if self.h:
            self.lib.spires_reservoir_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, u=None):
        p = None if u is None else dptr(np.ascontiguousarray(u, dtype=np.float64))
        st = self.lib.spires_step(self.h, p)
        assert st == SPIRES_OK, st

    def reset(self):
        assert self.lib.spires_reservoir_reset(self.h) == SPIRES_OK

    def state(self):
        v = np.empty(self.n)
        assert self.lib.spires_read_reservoir_state(self.h, dptr(v)) == SPIRES_OK
        return v

    def spikes(self):
        v = np.empty(self.n)
        assert self.lib.spires_read_spike_state(self.h, dptr(v)) == SPIRES_OK
        return v

    def weights(self):
        w = np.empty(self.n * self.n)
        assert self.lib.spires_read_weights(self.h, dptr(w)) == SPIRES_OK
        return w.reshape(self.n, self.n)

    def readout(self):
        w = np.empty(self.n * self.dout)
        assert self.lib.spires_read_readout(self.h, dptr(w)) == SPIRES_OK
        return w.reshape(self.dout, self.n)

    def output(self):
        y = np.empty(max(self.dout, 1))
        assert self.lib.spires_compute_output(self.h, dptr(y)) == SPIRES_OK
        return y[: self.dout]

    def run(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        T = u.shape[0]
        p = self.lib.spires_run(self.h, dptr(u), T)
        assert p, "spires_run returned NULL"
        y = np.ctypeslib.as_array(p, shape=(T * self.dout,)).copy()
        libc.free(C.cast(p, C.c_void_p))
        return y.reshape(T, self.dout)

    def train_ridge(self, u, y, lam):
        u = np.ascontiguousarray(u, dtype=np.float64)
        y = np.ascontiguousarray(y, dtype=np.float64)
        st = self.lib.spires_train_ridge(self.h, dptr(u), dptr(y), u.shape[0], lam)
        assert st == SPIRES_OK, st

    def train_rls(self, u, y, delta, lam):
        u = np.ascontiguousarray(u, dtype=np.float64)
        y = np.ascontiguousarray(y, dtype=np.float64)
        st = self.lib.spires_train_rls(self.h, dptr(u), dptr(y), u.shape[0], delta, lam)
        assert st == SPIRES_OK, st

    def train_online(self, target, lr):
        t = np.ascontiguousarray(target, dtype=np.float64)
        assert self.lib.spires_train_online(self.h, dptr(t), lr) == SPIRES_OK

    # ---- extensions (this library only)
    def run_record(self, u, T=None, phi=True, raster=True, y=False):
        if u is not None:
            u = np.ascontiguousarray(u, dtype=np.float64)
            T = u.shape[0]
        nw = (self.n + 31) // 32
        P = np.empty((T, self.n)) if phi else None
        R = np.empty((T, nw), dtype=np.uint32) if raster else None
        Y = np.empty((T, max(self.dout, 1))) if y else None
        st = self.lib.spires_ext_run_record(
            self.h, None if u is None else dptr(u), T, None if P is None else dptr(P),
            None if R is None else R.ctypes.data_as(_u32p), None if Y is None else dptr(Y))
        assert st == SPIRES_OK, st
        return P, R, Y

    def set_weights(self, dense, rescale=True):
        """spires_ext_set_weights: dense [n, n] recurrent weights (0 = no edge)."""
        d = np.ascontiguousarray(dense, np.float64)
        assert d.shape == (self.n, self.n)
        st = self.lib.spires_ext_set_weights(self.h, dptr(d), int(rescale))
        assert st == SPIRES_OK, st

    def w_in(self):
        w = np.empty(self.n * self.din)
        assert self.lib.spires_ext_read_w_in(self.h, dptr(w)) == SPIRES_OK
        return w.reshape(self.n, self.din)

    def launch(self):
        l = Launch()
        assert self.lib.spires_ext_get_launch(self.h, C.byref(l)) == SPIRES_OK
        return l

    def set_launch(self, **kw):
        l = self.launch()
        for k, v in kw.items():
            setattr(l, k, v)
        return self.lib.spires_ext_set_launch(self.h, C.byref(l))


class HostModel:
    """spires_ext_model: construction only, no GPU."""

    def __init__(self, cfg: Config, seed: int | None = None, lib: C.CDLL | None = None,
                 private: bool = False):
        """private=True draws from a private generator with the srand(seed) +
        rand() sequence instead of seeding the global one."""
        self.lib = lib or load()
        h = C.c_void_p()
        if private:
            st = self.lib.spires_ext_model_build_seeded(C.byref(cfg), int(seed or 0) & 0xFFFFFFFF,
                                                        C.byref(h))
        else:
            if seed is not None:
                libc.srand(seed)
            st = self.lib.spires_ext_model_build(C.byref(cfg), C.byref(h))
        if st != SPIRES_OK:
            raise RuntimeError(f"spires_ext_model_build failed: {st}")
        self.h = h
        info = ModelInfo()
        self.lib.spires_ext_model_info_get(h, C.byref(info))
        self.info = info
        self.n = int(info.num_neurons)

    def __del__(self):
        try:
            if self.h:
                self.lib.spires_ext_model_free(self.h)
        except Exception:
            pass

    def csr(self):
        n, nnz = self.n, int(self.info.nnz)
        rp = np.empty(n + 1, np.int64)
        col = np.empty(max(nnz, 1), np.int32)
        val = np.empty(max(nnz, 1))
        self.lib.spires_ext_model_csr(self.h, rp.ctypes.data_as(_i64p),
                                      col.ctypes.data_as(_i32p), dptr(val))
        return rp, col[:nnz], val[:nnz]

    def dense(self):
        rp, col, val = self.csr()
        W = np.zeros((self.n, self.n))
        rows = np.repeat(np.arange(self.n), np.diff(rp))
        W[rows, col] = val
        return W

    def w_in(self):
        w = np.empty(self.n * int(self.info.num_inputs))
        self.lib.spires_ext_model_w_in(self.h, dptr(w))
        return w.reshape(self.n, -1)

    def w_out(self):
        w = np.empty(self.n * int(self.info.num_outputs))
        self.lib.spires_ext_model_w_out(self.h, dptr(w))
        return w.reshape(-1, self.n)

    def edge_tau(self):
        t = np.empty(max(int(self.info.nnz), 1))
        self.lib.spires_ext_model_edge_tau(self.h, dptr(t))
        return t[: int(self.info.nnz)]

    def coef(self):
        c = np.empty(max(self.info.ring_len, 1))
        self.lib.spires_ext_model_coef(self.h, dptr(c))
        return c


class Batch:
    """spires_ext_batch: many reservoirs simulated in one persistent launch.

    cfgs: list of Config; seeds: one srand() seed per instance (instance k is
    built as spires_reservoir_create after srand(seeds[k]))."""

    def __init__(self, cfgs, seeds, lib: C.CDLL | None = None):
        self.lib = lib or load()
        self.count = len(cfgs)
        arr = (Config * self.count)()
        for k, c in enumerate(cfgs):
            arr[k] = c
        self._cfgs = list(cfgs)  # keeps parameter arrays alive
        sd = (C.c_uint * self.count)(*[int(x) & 0xFFFFFFFF for x in seeds])
        h = C.c_void_p()
        st = self.lib.spires_ext_batch_create(arr, sd, self.count, C.byref(h))
        if st != SPIRES_OK:
            raise RuntimeError(f"spires_ext_batch_create failed: {st}")
        self.h = h
        self.n = [int(c.num_neurons) for c in cfgs]
        self.din = [int(c.num_inputs) for c in cfgs]
        self.dout = [int(c.num_outputs) for c in cfgs]

    def close(self):
        if self.h:
            self.lib.spires_ext_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _inputs(self, us, T):
        if us is None:
            return None, [int(t) for t in T], []
        keep = [np.ascontiguousarray(u, dtype=np.float64) for u in us]
        T = [u.shape[0] for u in keep] if T is None else [int(t) for t in T]
        ptrs = (_dp * self.count)(*[dptr(u) for u in keep])
        return ptrs, T, keep

    def run(self, us=None, T=None, rasters=True, states=True):
        """Run every instance from reset; returns (rasters, final states, device ms)."""
        up, T, keep = self._inputs(us, T)
        Ts = (C.c_size_t * self.count)(*T)
        R = [np.empty((T[k], (self.n[k] + 31) // 32), np.uint32) for k in range(self.count)] \
            if rasters else None
        V = [np.empty(self.n[k]) for k in range(self.count)] if states else None
        rp = (_u32p * self.count)(*[r.ctypes.data_as(_u32p) for r in R]) if R else None
        vp = (_dp * self.count)(*[dptr(v) for v in V]) if V else None
        ms = C.c_double(0.0)
        st = self.lib.spires_ext_batch_run(self.h, up, Ts, rp, vp, C.byref(ms))
        if st != SPIRES_OK:
            raise RuntimeError(f"spires_ext_batch_run failed: {st}")
        return R, V, ms.value

    def train_ridge(self, us, ys, lam, washout=0, gram_mode=0, T=None):
        """Ridge readout of every instance; returns (list of W_out [dout, n], wall ms)."""
        up, T, keep = self._inputs(us, T)
        ykeep = [np.ascontiguousarray(y, dtype=np.float64) for y in ys]
        yp = (_dp * self.count)(*[dptr(y) for y in ykeep])
        Ts = (C.c_size_t * self.count)(*T)
        lams = np.ascontiguousarray(np.broadcast_to(np.asarray(lam, np.float64), (self.count,)))
        W = [np.empty((self.dout[k], self.n[k])) for k in range(self.count)]
        wp = (_dp * self.count)(*[dptr(w) for w in W])
        o = RidgeOpts(gram_mode, 30, 1e-13, washout)
        ms = C.c_double(0.0)
        st = self.lib.spires_ext_batch_train_ridge(self.h, up, yp, Ts, dptr(lams), C.byref(o),
                                                   wp, C.byref(ms))
        if st != SPIRES_OK:
            raise RuntimeError(f"spires_ext_batch_train_ridge failed: {st}")
        return W, ms.value

    def predict(self, us, T=None):
        """Readouts of every instance from reset with its current W_out."""
        up, T, keep = self._inputs(us, T)
        Ts = (C.c_size_t * self.count)(*T)
        Y = [np.empty((T[k], max(self.dout[k], 1))) for k in range(self.count)]
        yp = (_dp * self.count)(*[dptr(y) for y in Y])
        ms = C.c_double(0.0)
        st = self.lib.spires_ext_batch_predict(self.h, up, Ts, yp, C.byref(ms))
        if st != SPIRES_OK:
            raise RuntimeError(f"spires_ext_batch_predict failed: {st}")
        return Y, ms.value

    def fit_predict(self, us, ys, T_fit, lam, washout=0, gram_mode=0):
        """One simulation of every full series: ridge on rows [washout, T_fit[k]),
        readouts of all rows returned (list of [T_k, dout_k])."""
        up, T, keep = self._inputs(us, None)
        ykeep = [np.ascontiguousarray(y, dtype=np.float64) for y in ys]
        yp = (_dp * self.count)(*[dptr(y) for y in ykeep])
        Ts = (C.c_size_t * self.count)(*T)
        Tf = (C.c_size_t * self.count)(*[int(t) for t in T_fit])
        lams = np.ascontiguousarray(np.broadcast_to(np.asarray(lam, np.float64), (self.count,)))
        Y = [np.empty((T[k], max(self.dout[k], 1))) for k in range(self.count)]
        op = (_dp * self.count)(*[dptr(v) for v in Y])
        o = RidgeOpts(gram_mode, 30, 1e-13, washout)
        ms = C.c_double(0.0)
        st = self.lib.spires_ext_batch_fit_predict(self.h, up, yp, Ts, Tf, dptr(lams), C.byref(o),
                                                   op, None, C.byref(ms))
        if st != SPIRES_OK:
            raise RuntimeError(f"spires_ext_batch_fit_predict failed: {st}")
        return Y, ms.value

    def timing(self):
        """(construct_ms, setup_ms) of the batch's creation."""
        a, b = C.c_double(), C.c_double()
        self.lib.spires_ext_batch_timing(self.h, C.byref(a), C.byref(b))
        return a.value, b.value

    def info(self):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        self.lib.spires_ext_batch_info(self.h, C.byref(a), C.byref(b), C.byref(c))
        return {"ctas": a.value, "groups": b.value, "graph": c.value}

    def autotune(self, us=None, T=None):
        """spires_ext_batch_autotune over a sample of the series: returns the
        chosen schedule family, grid size and device ms."""
        up, T, keep = self._inputs(us, T)
        Ts = (C.c_size_t * self.count)(*T)
        mode, ctas, ms = C.c_int(), C.c_int(), C.c_double()
        st = self.lib.spires_ext_batch_autotune(self.h, up, Ts, C.byref(mode), C.byref(ctas),
                                                C.byref(ms))
        if st != SPIRES_OK:
            raise RuntimeError(f"spires_ext_batch_autotune failed: {st}")
        return {"schedule": mode.value, "ctas": ctas.value, "ms": ms.value}


def ridge_fit(states, targets, lam, washout=0, gram_mode=0, max_refine=30, lib=None):
    """spires_ext_ridge_fit: W_out [dout, n] from host states/targets, and the report."""
    lib = lib or load()
    X = np.ascontiguousarray(states, np.float64)
    Y = np.ascontiguousarray(targets, np.float64)
    if Y.ndim == 1:
        Y = Y[:, None]
    W = np.empty((Y.shape[1], X.shape[1]))
    o = RidgeOpts(gram_mode, max_refine, 1e-13, washout)
    rep = RidgeReport()
    st = lib.spires_ext_ridge_fit(dptr(X), X.shape[0], X.shape[1], dptr(Y), Y.shape[1], lam,
                                  C.byref(o), dptr(W), C.byref(rep))
    if st != SPIRES_OK:
        raise RuntimeError(f"spires_ext_ridge_fit failed: {st}")
    return W, rep


def fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_fp)


class Surrogate:
    """spires_ext_mlp: the 10 -> 128 -> 128 -> 2 surrogate on the GPU."""

    IN = 10

    def __init__(self, seed: int = 0, lib: C.CDLL | None = None):
        self.lib = lib or load()
        h = C.c_void_p()
        st = self.lib.spires_ext_mlp_create(seed, C.byref(h))
        if st != SPIRES_OK:
            raise RuntimeError(f"spires_ext_mlp_create failed: {st}")
        self.h = h
        self.num_params = int(self.lib.spires_ext_mlp_num_params())

    def close(self):
        if self.h:
            self.lib.spires_ext_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        p = np.empty(self.num_params, np.float32)
        assert self.lib.spires_ext_mlp_get_params(self.h, fptr(p)) == SPIRES_OK
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert self.lib.spires_ext_mlp_set_params(self.h, fptr(p)) == SPIRES_OK

    def loss_grad(self, X, y):
        X = np.ascontiguousarray(X, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        loss = np.zeros(1, np.float32)
        g = np.empty(self.num_params, np.float32)
        st = self.lib.spires_ext_mlp_loss_grad(self.h, fptr(X), fptr(y), X.shape[0], fptr(loss),
                                               fptr(g))
        assert st == SPIRES_OK, st
        return float(loss[0]), g

    def train(self, X, y, epochs=50, batch=256, lr=1e-3, seed=0):
        X = np.ascontiguousarray(X, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        loss = np.zeros(1, np.float32)
        st = self.lib.spires_ext_mlp_train(self.h, fptr(X), fptr(y), X.shape[0], epochs, batch,
                                           lr, seed, fptr(loss))
        assert st == SPIRES_OK, st
        return float(loss[0])

    def predict(self, X, bf16=True):
        X = np.ascontiguousarray(X, np.float32)
        m = np.empty(X.shape[0], np.float32)
        v = np.empty(X.shape[0], np.float32)
        st = self.lib.spires_ext_mlp_predict(self.h, fptr(X), X.shape[0], int(bf16), fptr(m),
                                             fptr(v))
        assert st == SPIRES_OK, st
        return m, v


def unpack_raster(R: np.ndarray, n: int) -> np.ndarray:
    """[T, nwords] uint32 spike words -> [T, n] uint8 (bit i%32 of word i/32)."""
    b = np.unpackbits(R.view(np.uint8).reshape(R.shape[0], -1), axis=1, bitorder="little")
    return b[:, :n]
