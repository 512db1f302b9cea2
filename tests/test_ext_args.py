"""The extension entry points (include/spires_ext.h) check their arguments
before any device work: missing handles, buffers and out-of-range sizes give
SPIRES_ERR_INVALID_ARG, destroy(NULL) is a no-op, and the host power
iteration computes what its definition says. Runs on the CPU only."""
import ctypes as C

import numpy as np

import spires_b200 as sp
from oracle import surrogate_oracle as SO

INVALID = sp.SPIRES_ERR_INVALID_ARG


def lib():
    return sp.load()


def test_destroy_null_is_safe():
    L = lib()
    L.spires_ext_batch_destroy(None)
    L.spires_ext_mlp_destroy(None)
    L.spires_ext_model_free(None)
    L.spires_ext_agile_batch_destroy(None)
    assert L.spires_ext_mlp_kernel_launches(None) == 0


def test_batch_calls_reject_missing_arguments():
    L = lib()
    out = C.c_void_p()
    cfg = sp.make_config(64)
    seeds = (C.c_uint * 1)(1)
    assert L.spires_ext_batch_create(None, seeds, 1, C.byref(out)) == INVALID
    assert L.spires_ext_batch_create(C.byref(cfg), seeds, 0, C.byref(out)) == INVALID
    assert L.spires_ext_batch_create(C.byref(cfg), seeds, 1, None) == INVALID
    T = (C.c_size_t * 1)(10)
    assert L.spires_ext_batch_run(None, None, T, None, None, None) == INVALID
    assert L.spires_ext_batch_train_ridge(None, None, None, T, None, None, None, None) == INVALID
    assert L.spires_ext_batch_predict(None, None, T, None, None) == INVALID
    assert L.spires_ext_batch_fit_predict(None, None, None, T, T, None, None, None, None,
                                          None) == INVALID
    assert L.spires_ext_batch_info(None, None, None, None) == INVALID
    assert L.spires_ext_batch_timing(None, None, None) == INVALID


def test_mlp_calls_reject_missing_arguments():
    L = lib()
    assert L.spires_ext_mlp_num_params() == SO.NUM_PARAMS
    assert L.spires_ext_mlp_create(1, None) == INVALID
    buf = (C.c_float * 4)()
    assert L.spires_ext_mlp_get_params(None, buf) == INVALID
    assert L.spires_ext_mlp_set_params(None, buf) == INVALID
    assert L.spires_ext_mlp_loss_grad(None, buf, buf, 1, buf, buf) == INVALID
    assert L.spires_ext_mlp_train(None, buf, buf, 1, 1, 1, 1e-3, 0, None) == INVALID
    assert L.spires_ext_mlp_predict(None, buf, 1, 0, buf, buf) == INVALID


def test_ridge_fit_rejects_bad_sizes():
    L = lib()
    X = np.zeros((8, 4))
    Y = np.zeros((8, 2))
    W = np.zeros((2, 4))
    o = sp.RidgeOpts(0, 30, 1e-13, 0)
    assert L.spires_ext_ridge_fit(None, 8, 4, sp.dptr(Y), 2, 1.0, None, sp.dptr(W),
                                  None) == INVALID
    for n, dout in ((0, 2), (4, 0)):
        assert L.spires_ext_ridge_fit(sp.dptr(X), 8, n, sp.dptr(Y), dout, 1.0, None,
                                      sp.dptr(W), None) == INVALID
    o.washout = 8  # nothing left after the washout
    assert L.spires_ext_ridge_fit(sp.dptr(X), 8, 4, sp.dptr(Y), 2, 1.0, C.byref(o), sp.dptr(W),
                                  None) == INVALID


def test_noalloc_ridge_rejects_before_touching_the_device():
    L = lib()
    p = C.c_void_p(1)  # never dereferenced: the size checks come first
    assert L.spires_ext_ridge_solve_noalloc(None, p, 10, 4, 1, 0, 1.0, p, None) == INVALID
    assert L.spires_ext_ridge_solve_noalloc(p, p, 10, 4, 1, 10, 1.0, p, None) == INVALID
    assert L.spires_ext_ridge_solve_noalloc(p, p, 10, 513, 1, 0, 1.0, p, None) == INVALID
    assert L.spires_ext_ridge_solve_noalloc(p, p, 10, 4, 17, 0, 1.0, p, None) == INVALID
    assert L.spires_ext_ridge_solve_noalloc(p, p, 16385, 4, 1, 0, 1.0, p, None) == INVALID


def test_model_and_weights_calls_reject_missing_arguments():
    L = lib()
    out = C.c_void_p()
    assert L.spires_ext_model_build_seeded(None, 1, C.byref(out)) == INVALID
    assert L.spires_ext_model_build_seeded(C.byref(sp.make_config(10)), 1, None) == INVALID
    d = np.zeros(4)
    assert L.spires_ext_set_weights(None, sp.dptr(d), 0) == INVALID
    val = C.c_double()
    assert L.spires_ext_spectral_radius(3, None, None, None, 0, C.byref(val)) == INVALID


def test_agile_batch_rejects_bad_shapes():
    L = lib()
    out = C.c_void_p()
    th = np.full(2, 0.5)
    lo = np.zeros(2)
    hi = np.ones(2)
    args = [sp.dptr(th), sp.dptr(lo), sp.dptr(hi)]
    for chains, dim in ((0, 2), (2, 0), (2, 65)):  # default options and seeds
        assert L.spires_ext_agile_batch_create(chains, dim, *args, None, None,
                                               C.byref(out)) == INVALID
    assert L.spires_ext_agile_batch_tell(None, sp.dptr(th)) == INVALID
    assert L.spires_ext_agile_batch_best(None, 0, sp.dptr(th), None) == INVALID


def power_iteration(n, rp, col, w):
    """csr_spectral_radius (src/sparse.c:93-127): max-abs normalised power
    iteration from x = 1, rows summed in edge order, tol 1e-6, 1000 steps."""
    x = [1.0] * n
    lam_old = lam = 0.0
    for _ in range(1000):
        y = []
        for i in range(n):
            s = 0.0
            for k in range(rp[i], rp[i + 1]):
                s += w[k] * x[col[k]]
            y.append(s)
        lam = max(abs(v) for v in y)
        x = [v / lam for v in y]
        if abs(lam - lam_old) < 1e-6:
            break
        lam_old = lam
    return lam


def test_host_spectral_radius_follows_its_definition():
    L = lib()
    rng = np.random.default_rng(3)
    n = 12
    A = rng.uniform(-1, 1, (n, n)) * (rng.uniform(0, 1, (n, n)) < 0.4)
    rp = np.zeros(n + 1, np.int64)
    rp[1:] = np.cumsum((A != 0).sum(axis=1))
    col = np.nonzero(A)[1].astype(np.int32)
    w = A[A != 0].astype(np.float64)
    out = C.c_double()
    st = L.spires_ext_spectral_radius(n, rp.ctypes.data_as(sp._i64p), col.ctypes.data_as(sp._i32p),
                                      sp.dptr(w), 0, C.byref(out))
    assert st == sp.SPIRES_OK
    assert out.value == power_iteration(n, list(rp), list(col), list(w))
