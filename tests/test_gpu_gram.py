"""Mixed-precision ridge: the Gram Phi^T Phi from split BF16 / TF32 operands
on the tensor cores (FP32 accumulation), FP64 Cholesky and iterative
refinement with residuals from the FP64 states, against the all-FP64 ridge on
the same states. Errors in W_out and in the readout's NRMSE are stated per
case; the refinement must reach the FP64 solution when the system is well
enough conditioned (lambda = 1e-3 here), to the stated residual."""
import ctypes as C

import numpy as np
import pytest

import spires_b200 as sp
from spires_b200.datasets import mackey_glass

pytestmark = pytest.mark.gpu

GL = (1.0, 0.0, 0.0, 20.0, 0.7, 128.0, 0.1, 2.0)


def fit(mode, lam, n=1000, T=4000, washout=200):
    cfg = sp.make_config(n, 1, 1, rho=0.95, ei=0.5, gamma=0.5, conn=10.0 / (n - 1),
                         topo=sp.CONN_SMALL_WORLD, neuron=sp.FLIF_GL, nparams=GL)
    x = mackey_glass(T + 1, seed=3)
    u, y = np.ascontiguousarray(x[:-1, None]), np.ascontiguousarray(x[1:, None])
    r = sp.Reservoir(cfg, seed=11)
    o = sp.RidgeOpts(mode, 300, 1e-13, washout)
    rep = sp.RidgeReport()
    st = r.lib.spires_ext_train_ridge(r.h, sp.dptr(u), sp.dptr(y), T, lam, C.byref(o),
                                      C.byref(rep))
    assert st == sp.SPIRES_OK
    W = r.readout()
    r.reset()
    yhat = r.run(u)
    r.close()
    e = yhat[washout:, 0] - y[washout:, 0]
    nrmse = float(np.sqrt(np.mean(e * e)) / y[washout:, 0].std())
    return W, nrmse, rep


@pytest.mark.parametrize("mode", [1, 2])
def test_split_gram_reaches_fp64_solution(mode):
    W64, n64, r64 = fit(0, 1e-3)
    W, nr, rep = fit(mode, 1e-3)
    assert rep.gram_mode_used == mode and r64.gram_mode_used == 0
    werr = np.linalg.norm(W - W64) / np.linalg.norm(W64)
    print(f"mode {mode} lambda 1e-3: W rel err {werr:.2e}, NRMSE {nr:.6f} vs {n64:.6f}, "
          f"refine {rep.refine_iters}, residual {rep.rel_residual:.1e}")
    # the conjugate-gradient refinement drives the FP64 residual down; W is
    # only determined up to the near-null space of the states, the readout's
    # predictions are
    assert rep.rel_residual < 1e-8
    assert werr < 1e-2
    assert abs(nr - n64) <= 1e-5 * n64


@pytest.mark.parametrize("mode", [1, 2])
def test_split_gram_small_lambda_stated_error(mode):
    W64, n64, _ = fit(0, 1e-6)
    W, nr, rep = fit(mode, 1e-6)
    werr = np.linalg.norm(W - W64) / np.linalg.norm(W64)
    print(f"mode {mode} lambda 1e-6: W rel err {werr:.2e}, NRMSE {nr:.6f} vs {n64:.6f}, "
          f"refine {rep.refine_iters}, residual {rep.rel_residual:.1e}")
    # ill-conditioned: the readout's NRMSE must still agree to 1 %
    assert np.isfinite(nr) and abs(nr - n64) <= 1e-2 * n64


@pytest.mark.parametrize("lam", [1e-3, 1e-6])
def test_int8_gram_ridge_is_the_fp64_ridge(lam):
    """INT8 integer-slice Gram (7 slices): as accurate as the FP64 Gram, so the
    same FP64 Cholesky and refinement reach a solution as close to an FP64
    LAPACK solve (numpy) of the same normal equations as the FP64-Gram path's.
    W itself is only determined to about cond(A) * eps (two FP64 solvers differ
    by that much); the fitted outputs agree tightly."""
    n, T, washout = 1000, 4000, 200
    W64, n64, r64 = fit(0, lam, n=n, T=T, washout=washout)
    W, nr, rep = fit(3, lam, n=n, T=T, washout=washout)
    assert rep.gram_mode_used == 3 and r64.gram_mode_used == 0
    assert rep.factor_failed == 0
    cfg = sp.make_config(n, 1, 1, rho=0.95, ei=0.5, gamma=0.5, conn=10.0 / (n - 1),
                         topo=sp.CONN_SMALL_WORLD, neuron=sp.FLIF_GL, nparams=GL)
    x = mackey_glass(T + 1, seed=3)
    u, y = np.ascontiguousarray(x[:-1, None]), np.ascontiguousarray(x[1:, None])
    r = sp.Reservoir(cfg, seed=11)
    phi, _, _ = r.run_record(u, raster=False)
    r.close()
    Xw = phi[washout:]
    A = Xw.T @ Xw
    A[np.diag_indices(n)] += lam
    Wnp = np.linalg.solve(A, Xw.T @ y[washout:]).T
    e8 = np.linalg.norm(W - Wnp) / np.linalg.norm(Wnp)
    e64 = np.linalg.norm(W64 - Wnp) / np.linalg.norm(Wnp)
    werr = np.linalg.norm(W - W64) / np.linalg.norm(W64)
    print(f"int8 lambda {lam:g}: W rel err vs LAPACK {e8:.2e} (fp64 Gram path {e64:.2e}), "
          f"vs fp64 path {werr:.2e}; NRMSE {nr:.9f} vs {n64:.9f}; residual "
          f"{rep.rel_residual:.1e} (fp64 {r64.rel_residual:.1e})")
    assert rep.rel_residual <= max(10 * r64.rel_residual, 1e-12)
    assert e8 <= 2 * e64 + 1e-12
    assert abs(nr - n64) <= 1e-8 * n64


def test_int8_gram_ridge_at_full_size_against_fp64():
    """FLIF_GL N=4000, L=512, Watts-Strogatz k=10, Mackey-Glass T=20000,
    washout 1000, lambda 1e-6: W_out and NRMSE of the INT8-Gram ridge and of
    the FP64-Gram ridge, each against an FP64 solve (numpy, LAPACK) of the
    same normal equations on the same states. Stated, and bounded by the
    FP64-Gram path's own distance to that solve."""
    n, T, w, lam = 4000, 20000, 1000, 1e-6
    cfg = sp.make_config(n, 1, 1, rho=0.95, ei=0.5, gamma=0.5, conn=10.0 / (n - 1),
                         topo=sp.CONN_SMALL_WORLD, neuron=sp.FLIF_GL,
                         nparams=(1.0, 0.0, 0.0, 20.0, 0.7, 512.0, 0.1, 2.0))
    x = mackey_glass(T + 1, seed=0)
    u, y = np.ascontiguousarray(x[:-1, None]), np.ascontiguousarray(x[1:, None])
    r = sp.Reservoir(cfg, seed=42)
    phi, _, _ = r.run_record(u, phi=True, raster=False)
    r.close()
    Xw = phi[w:]
    A = Xw.T @ Xw
    A[np.diag_indices(n)] += lam
    Wnp = np.linalg.solve(A, Xw.T @ y[w:]).T

    def nrmse(W):
        e = Xw @ W.T - y[w:]
        return float(np.sqrt(np.mean(e * e)) / y[w:, 0].std())

    out = {}
    for mode in (0, 3):
        W, rep = sp.ridge_fit(phi, y, lam, washout=w, gram_mode=mode, max_refine=30)
        out[mode] = (float(np.linalg.norm(W - Wnp) / np.linalg.norm(Wnp)),
                     abs(nrmse(W) - nrmse(Wnp)) / nrmse(Wnp), rep.refine_iters,
                     rep.rel_residual, rep.gram_ms)
        print(f"mode {mode}: W rel err vs numpy FP64 {out[mode][0]:.2e}, NRMSE rel err "
              f"{out[mode][1]:.2e}, refine {out[mode][2]}, residual {out[mode][3]:.1e}, "
              f"Gram {out[mode][4]:.1f} ms")
    assert out[3][0] <= max(2 * out[0][0], 1e-6)
    assert out[3][1] <= max(2 * out[0][1], 1e-9)
