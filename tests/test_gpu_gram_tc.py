"""The tensor-core Gram (spires_b200/csrc/gram_tc.cu) through
spires_ext_gram_device.

* INT8 slices: bit for bit the model of tests/_ozaki_model.py (exact int32
  level sums, the same FP64 combination order), for several slice counts,
  ragged sizes (n and T not multiples of the tiles), a washout offset, a zero
  column, columns of very different magnitudes, and more rows than one
  int32-safe segment; and within FP64-dgemm accuracy of the exact Gram.
* BF16X3 / TF32X3 splits: within their FP32-accumulation error bound of the
  FP64 Gram.
* FP64 mode: the CUDA-core SYRK of the ridge solver.
The reference forms this Gram with one cblas_dgemm (src/math_utils.c:154-162,
called from src/reservoir.c:615-623)."""
import ctypes as C

import numpy as np
import pytest

import spires_b200 as sp
from tests import _ozaki_model as M

pytestmark = pytest.mark.gpu


def gram_dev(X, mode, slices=0, t0=0):
    import torch

    lib = sp.load()
    T, n = X.shape
    dX = torch.from_numpy(np.ascontiguousarray(X)).cuda()
    dC = torch.full((n, n), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    st = lib.spires_ext_gram_device(C.c_void_p(dX.data_ptr()), T, n, t0, mode, slices,
                                    C.c_void_p(dC.data_ptr()), None)
    assert st == sp.SPIRES_OK, st
    return dC.cpu().numpy()


def states(T, n, seed, scale_cols=False):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((T, n)) * rng.uniform(0.1, 2.0, n)[None, :]
    if scale_cols:
        X[:, 0] *= 1e-30
        X[:, 1] *= 1e30
        X[:, 2] = 0.0
    return X


@pytest.mark.parametrize("T,n,slices,t0", [(300, 100, 7, 0), (1000, 257, 7, 13),
                                           (777, 130, 8, 0), (500, 64, 4, 0),
                                           (2048, 384, 6, 100)])
def test_int8_gram_is_the_model_bit_for_bit(T, n, slices, t0):
    X = states(T, n, seed=T + n, scale_cols=True)
    G = gram_dev(X, 3, slices, t0)
    Gm = M.ozaki_gram(X[t0:], slices)
    assert np.array_equal(G.view(np.uint64), Gm.view(np.uint64))
    assert np.array_equal(G, G.T)


def test_int8_gram_segments():
    """More rows than one int32-safe segment (65472): segment Grams are added
    in order, as the model does."""
    X = states(70000, 40, seed=5)
    G = gram_dev(X, 3, 7)
    Gm = M.ozaki_gram(X, 7)
    assert np.array_equal(G.view(np.uint64), Gm.view(np.uint64))


def test_int8_gram_accuracy_matches_fp64():
    X = states(4000, 200, seed=9)
    Xl = X.astype(np.longdouble)
    Gx = (Xl.T @ Xl)
    den = (np.abs(X).T @ np.abs(X))

    def err(G):
        return float(np.max(np.abs(G.astype(np.longdouble) - Gx) / den))

    e64 = err(gram_dev(X, 0))
    e7 = err(gram_dev(X, 3, 7))
    e8 = err(gram_dev(X, 3, 8))
    assert e64 < 1e-14
    assert e7 < 4 * e64 + 1e-16
    assert e8 <= e64 + 1e-17


# FP32 accumulation over 1500 rows: the split products' rounding (2^-16 for
# BF16 hi/lo, 2^-22 for TF32) plus the sums' own, relative to |X|^T |X|
@pytest.mark.parametrize("mode,tol", [(1, 2e-4), (2, 1e-4)])
def test_split_grams_within_fp32_bound(mode, tol):
    X = states(1500, 190, seed=3)
    G = gram_dev(X, mode)
    G64 = X.T @ X
    den = np.abs(X).T @ np.abs(X)
    assert np.max(np.abs(G - G64) / den) < tol
    assert np.array_equal(G, G.T)


def test_fp64_gram_mode():
    X = states(900, 150, seed=4)
    G = gram_dev(X, 0)
    assert np.allclose(G, X.T @ X, rtol=1e-13, atol=1e-13 * np.abs(X.T @ X).max())
