"""Model of the tensor-core Gram of the ridge readout (test infrastructure).

Restates, in numpy, the arithmetic of spires_b200/csrc/gram_tc.cu so the
device result can be checked bit for bit:

* integer-slice Gram (Ozaki, Ogita, Oishi, Rump, "Error-free transformations of
  matrix multiplication by using fast routines of matrix multiplication and its
  applications", Numer. Algorithms 59, 2012, with int8 slices): each state
  column i is scaled by 2^-e_i (max_t |x_ti| < 2^e_i), then cut into k signed
  digits d_1..d_k, |d_s| <= 64, with x = sum_s d_s 2^(-6-7(s-1)) + r and
  |r| <= 2^-7k; the Gram is sum over pairs s + u <= k + 1 of d_s^T d_u scaled by
  2^(-12-7(s+u-2)). The pairs of one level s + u are summed exactly (int32 on
  the device, exact integers in FP64 here); the k level sums are combined in
  FP64 from the smallest level up, then scaled by 2^(e_i + e_j - 12). Rows are
  taken in segments of at most 65472 so no level sum can leave int32; segment
  Grams are added in order.
* split Gram: x = hi + lo (BF16 or TF32 roundings), G = hi^T hi + hi^T lo +
  lo^T hi accumulated in FP32 (the model only bounds this one; FP32
  accumulation order on the tensor cores is not specified).
"""
import numpy as np

SEG_ROWS = 65472


def column_exponents(X):
    amax = np.abs(X).max(axis=0) if X.shape[0] else np.zeros(X.shape[1])
    _, e = np.frexp(amax)
    return np.where(amax > 0, e, 0).astype(np.int64)


def digits(X, e, k):
    x = np.ldexp(X, -e[None, :])
    v = x * 64.0
    out = []
    for _ in range(k):
        d = np.rint(v)
        out.append(d)
        v = (v - d) * 128.0
    return out


def ozaki_gram(X, k=8):
    """Gram X^T X of the device's integer-slice mode (k slices)."""
    X = np.asarray(X, np.float64)
    T, n = X.shape
    e = column_exponents(X)
    G = None
    for t0 in range(0, max(T, 1), SEG_ROWS):
        D = digits(X[t0:t0 + SEG_ROWS], e, k)
        v = np.zeros((n, n))
        for lvl in reversed(range(k)):
            acc = np.zeros((n, n))
            for s in range(1, lvl + 2):
                u = lvl + 2 - s
                acc += D[s - 1].T @ D[u - 1]  # integers below 2^53: exact
            v = v + acc * 2.0 ** (-7 * lvl)
        Gs = np.ldexp(v, e[:, None] + e[None, :] - 12)
        G = Gs if G is None else G + Gs
    return G


def ozaki_error_bound(X, k=8):
    """Elementwise bound on |G_ozaki - X^T X| from the dropped digit pairs and
    the digit remainders (before the FP64 combination's own rounding)."""
    X = np.asarray(X, np.float64)
    T = X.shape[0]
    e = column_exponents(X)
    scale = np.ldexp(np.ones((X.shape[1], X.shape[1])), e[:, None] + e[None, :])
    # per row: |x_i x_j - sum_kept| <= (2 (k+1) + 1) 2^-7k for |x|<1 (loose)
    return scale * T * (2 * k + 3) * 2.0 ** (-7 * k)
