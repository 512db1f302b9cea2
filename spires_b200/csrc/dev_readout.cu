// dev_readout.cu -- readout training on the device.
//
//   ridge  (src/reservoir.c:573-679): reset, record Phi[T][N] (no washout unless
//          asked), A = Phi^T Phi + lambda I, B = Phi^T Y, solve A W = B.
//          The reference forms A with dgemm and solves one LU (dgesv) per
//          output; here A is factored once by a blocked Cholesky in FP64 and
//          all outputs are solved together, followed by iterative refinement
//          whose residual R = Phi^T (Y - Phi W) - lambda W is formed from the
//          FP64 Phi itself. A non-positive pivot falls back to LU with partial
//          pivoting, which is what dgesv does.
//   RLS    (src/reservoir.c:681-767) and the online delta rule
//          (src/reservoir.c:244-280), with W_out and P resident on the device.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <chrono>
#include "sp_alloc.h"
#include "sp_dev.h"
#include "sp_kernels.cuh"
#include "sp_dev_internal.h"
#include "sp_gram.h"

using namespace sp;

#define RK(x)                                                                      \
    do {                                                                           \
        cudaError_t e_ = (x);                                                      \
        if (e_ != cudaSuccess) {                                                   \
            sp_dev_note_error(#x, e_);                                             \
            rc = (e_ == cudaErrorMemoryAllocation) ? SP_EALLOC : SP_EINTERNAL;     \
            goto out;                                                              \
        }                                                                          \
    } while (0)

namespace {

constexpr int NB = 64;  // Cholesky panel width

// ---------------------------------------------------------------- Gram (FP64)
// C = X^T X over rows [t0, t1) of X (T x n, row-major); lower tiles computed,
// the upper triangle mirrored. 64x64 tile per CTA, 4x4 per thread.
__global__ void __launch_bounds__(256) k_syrk_f64(const double *__restrict__ X, int n, size_t t0,
                                                  size_t t1, double *__restrict__ C, int ldc)
{
    // tile index -> (bi, bj) with bi >= bj
    int b = blockIdx.x;
    int bi = (int)((sqrt(8.0 * b + 1.0) - 1.0) * 0.5);
    while ((bi + 1) * (bi + 2) / 2 <= b) ++bi;
    while (bi * (bi + 1) / 2 > b) --bi;
    int bj = b - bi * (bi + 1) / 2;
    const int i0 = bi * 64, j0 = bj * 64;
    __shared__ double si[16][64 + 1];
    __shared__ double sj[16][64 + 1];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    double acc[4][4] = {};
    for (size_t t = t0; t < t1; t += 16) {
        for (int q = threadIdx.x; q < 16 * 64; q += 256) {
            int r = q >> 6, c = q & 63;
            size_t tt = t + r;
            si[r][c] = (tt < t1 && i0 + c < n) ? X[tt * n + i0 + c] : 0.0;
            sj[r][c] = (tt < t1 && j0 + c < n) ? X[tt * n + j0 + c] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            double a[4], bb[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                a[u] = si[r][ty * 4 + u];
                bb[u] = sj[r][tx * 4 + u];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v)
                    acc[u][v] = fma(a[u], bb[v], acc[u][v]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            int i = i0 + ty * 4 + u, j = j0 + tx * 4 + v;
            if (i < n && j < n && j <= i) {
                C[(size_t)i * ldc + j] = acc[u][v];
                C[(size_t)j * ldc + i] = acc[u][v];
            }
        }
}

// R[i][o] = sum_{t in [t0,t1)} X[t][i] E[t][o] (- lam * W[i][o] when W != 0),
// split over `parts` contiguous t ranges reduced in a fixed order.
__global__ void k_xt_e_part(const double *__restrict__ X, int n, size_t t0, size_t t1,
                            const double *__restrict__ E, int dout, int parts,
                            double *__restrict__ part)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int pidx = blockIdx.y;
    const size_t len = t1 - t0;
    const size_t a = t0 + len * pidx / parts, b = t0 + len * (pidx + 1) / parts;
    if (i >= n)
        return;
    double acc[16];
    for (int o = 0; o < dout; ++o)
        acc[o] = 0.0;
    for (size_t t = a; t < b; ++t) {
        double x = X[t * n + i];
        for (int o = 0; o < dout; ++o)
            acc[o] = fma(x, E[t * dout + o], acc[o]);
    }
    for (int o = 0; o < dout; ++o)
        part[((size_t)pidx * n + i) * dout + o] = acc[o];
}

__global__ void k_reduce_parts(const double *__restrict__ part, int parts, int n, int dout,
                               const double *__restrict__ W, double lam, double *__restrict__ R)
{
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t total = (size_t)n * dout;
    if (k >= total)
        return;
    double s = 0.0;
    for (int p = 0; p < parts; ++p)
        s += part[(size_t)p * total + k];
    if (W)
        s -= lam * W[k];
    R[k] = s;
}

// E[t][o] = Y[t][o] - sum_i X[t][i] W[i][o], one warp per row t.
__global__ void k_resid_rows(const double *__restrict__ X, int n, size_t t0, size_t t1,
                             const double *__restrict__ Y, const double *__restrict__ W,
                             int dout, double *__restrict__ E)
{
    const size_t t = t0 + (size_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (t >= t1)
        return;
    double acc[16];
    for (int o = 0; o < dout; ++o)
        acc[o] = 0.0;
    for (int i = lane; i < n; i += 32) {
        double x = X[t * n + i];
        for (int o = 0; o < dout; ++o)
            acc[o] = fma(x, W[(size_t)i * dout + o], acc[o]);
    }
    for (int o = 0; o < dout; ++o) {
        double s = acc[o];
        for (int off = 16; off; off >>= 1)
            s += __shfl_xor_sync(kFull, s, off);
        if (lane == 0)
            E[t * dout + o] = Y[t * dout + o] - s;
    }
}

// Pt[k][t - t0] = X[t][k] for rows [t0, t1) of X (T x n): 32 x 32 tiles
// through shared memory, both sides coalesced.
__global__ void k_rows_to_cols(const double *__restrict__ X, int n, size_t t0, size_t t1,
                               double *__restrict__ Pt)
{
    __shared__ double tile[32][33];
    const size_t tw = t1 - t0;
    const size_t tb = (size_t)blockIdx.y * 32, kb = (size_t)blockIdx.x * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const size_t t = tb + r, k = kb + threadIdx.x;
        tile[r][threadIdx.x] = (t < tw && k < (size_t)n) ? X[(t0 + t) * n + k] : 0.0;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const size_t k = kb + r, t = tb + threadIdx.x;
        if (k < (size_t)n && t < tw)
            Pt[k * tw + t] = tile[threadIdx.x][r];
    }
}

__global__ void k_add_diag(double *A, int n, int lda, double lam)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        A[(size_t)i * lda + i] += lam;
}

// ------------------------------------------------------- blocked Cholesky
// A (n x n, row-major, lower triangle used) -> L in place.
// Diagonal block of panel [k0, k0 + kb), one CTA of 256 threads: thread t
// owns row t % 64 and the 16 columns t / 64 + 4 m of the trailing update.
// For column j every thread derives the factor itself from the current
// values (d = sqrt(a_jj), l_rj = a_rj / d as a_rj * (1 / d)) and updates its
// entries right of column j; the scaled column is written after the one
// barrier of the column, when nobody reads it any more.
__global__ void __launch_bounds__(256) k_potrf_diag(double *A, int n, int lda, int k0, int kb,
                                                    int *info)
{
    __shared__ double s[NB][NB + 1];
    __shared__ int bad;
    if (*info)
        return;
    for (int q = threadIdx.x; q < kb * kb; q += blockDim.x) {
        const int r = q / kb, c = q % kb;
        if (c <= r)
            s[r][c] = A[(size_t)(k0 + r) * lda + k0 + c];
    }
    if (threadIdx.x == 0)
        bad = 0;
    __syncthreads();
    const int r = threadIdx.x & (NB - 1), c0 = threadIdx.x >> 6;
    for (int j = 0; j < kb; ++j) {
        const double a = s[j][j];
        const bool okd = a > 0.0 && isfinite(a);
        const double d = okd ? sqrt(a) : 1.0;
        const double inv = 1.0 / d;
        double lrj = 0.0;
        if (r > j && r < kb) {
            lrj = s[r][j] * inv;
#pragma unroll
            for (int m = 0; m < NB / 4; ++m) {
                const int c = c0 + 4 * m;
                if (c > j && c <= r)
                    s[r][c] = fma(-lrj, s[c][j] * inv, s[r][c]);
            }
        }
        __syncthreads();  // every read of column j is done
        if (c0 == 0 && r > j && r < kb)
            s[r][j] = lrj;
        if (threadIdx.x == 0) {
            s[j][j] = d;
            if (!okd && !bad)
                bad = k0 + j + 1;
        }
    }
    __syncthreads();
    for (int q = threadIdx.x; q < kb * kb; q += blockDim.x) {
        const int rr = q / kb, cc = q % kb;
        if (cc <= rr)
            A[(size_t)(k0 + rr) * lda + k0 + cc] = s[rr][cc];
    }
    if (threadIdx.x == 0 && bad)
        atomicCAS(info, 0, bad);
}

// Rows r >= k0 + kb: L[r][k0:k0+kb] = A[r][k0:k0+kb] L_kk^-T. A warp solves 4
// rows side by side (independent chains), lane l holding columns l and l + 32
// of each; columns are eliminated in order (x_c = a_c * (1 / L_cc), then
// a_q -= x_c L_qc for q > c). 32 rows per CTA.
__global__ void __launch_bounds__(256) k_trsm_panel(double *A, int n, int lda, int k0, int kb,
                                                    const int *info)
{
    __shared__ double sL[NB][NB + 1];
    __shared__ double sInv[NB];
    if (*info)
        return;
    for (int q = threadIdx.x; q < kb * kb; q += blockDim.x) {
        const int r = q / kb, c = q % kb;
        sL[r][c] = (c <= r) ? A[(size_t)(k0 + r) * lda + k0 + c] : 0.0;
    }
    __syncthreads();
    if (threadIdx.x < kb)
        sInv[threadIdx.x] = 1.0 / sL[threadIdx.x][threadIdx.x];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r0 = k0 + kb + blockIdx.x * 32 + warp * 4;
    if (r0 >= n)
        return;
    double a0[4], a1[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const bool ok = r0 + q < n;
        const double *row = A + (size_t)(r0 + q) * lda + k0;
        a0[q] = ok && lane < kb ? row[lane] : 0.0;
        a1[q] = ok && lane + 32 < kb ? row[lane + 32] : 0.0;
    }
    for (int c = 0; c < kb; ++c) {
        const double ic = sInv[c];
        const double l0 = (lane > c && lane < kb) ? sL[lane][c] : 0.0;
        const double l1 = (lane + 32 > c && lane + 32 < kb) ? sL[lane + 32][c] : 0.0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const double xc = __shfl_sync(kFull, c < 32 ? a0[q] : a1[q], c & 31) * ic;
            if (lane == (c & 31)) {
                if (c < 32)
                    a0[q] = xc;
                else
                    a1[q] = xc;
            }
            if (lane > c && lane < kb)
                a0[q] = fma(-xc, l0, a0[q]);
            if (lane + 32 > c && lane + 32 < kb)
                a1[q] = fma(-xc, l1, a1[q]);
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        if (r0 + q >= n)
            break;
        double *row = A + (size_t)(r0 + q) * lda + k0;
        if (lane < kb)
            row[lane] = a0[q];
        if (lane + 32 < kb)
            row[lane + 32] = a1[q];
    }
}

// trailing update A22 -= L21 L21^T on lower tiles of the trailing matrix
__global__ void __launch_bounds__(256) k_syrk_update(double *A, int n, int lda, int k0, int kb,
                                                     const int *info)
{
    if (*info)
        return;
    const int base = k0 + kb;
    int b = blockIdx.x;
    int bi = (int)((sqrt(8.0 * b + 1.0) - 1.0) * 0.5);
    while ((bi + 1) * (bi + 2) / 2 <= b) ++bi;
    while (bi * (bi + 1) / 2 > b) --bi;
    int bj = b - bi * (bi + 1) / 2;
    const int i0 = base + bi * 64, j0 = base + bj * 64;
    __shared__ double si[64][33];
    __shared__ double sj[64][33];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    double acc[4][4] = {};
    for (int c0 = 0; c0 < kb; c0 += 32) {
        const int cw = (kb - c0 < 32) ? kb - c0 : 32;
        for (int q = threadIdx.x; q < 64 * 32; q += 256) {
            int r = q >> 5, c = q & 31;
            si[r][c] = (c < cw && i0 + r < n) ? A[(size_t)(i0 + r) * lda + k0 + c0 + c] : 0.0;
            sj[r][c] = (c < cw && j0 + r < n) ? A[(size_t)(j0 + r) * lda + k0 + c0 + c] : 0.0;
        }
        __syncthreads();
        for (int c = 0; c < cw; ++c) {
            double a[4], bb[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                a[u] = si[ty * 4 + u][c];
                bb[u] = sj[tx * 4 + u][c];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v)
                    acc[u][v] = fma(a[u], bb[v], acc[u][v]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            int i = i0 + ty * 4 + u, j = j0 + tx * 4 + v;
            if (i < n && j < n && j <= i)
                A[(size_t)i * lda + j] -= acc[u][v];
        }
}

// ----------------------------------------------------- triangular solves
// Forward L Z = B in place on Z (n x dout), panel by panel: the diagonal
// block by one CTA (warp w takes outputs w, w + 8, ...; lane l holds rows l
// and l + 32; columns eliminated in order, dividing by the diagonal as a
// product with its reciprocal), then the rows below it.
__global__ void __launch_bounds__(256) k_fwd_diag(const double *L, int lda, int k0, int kb,
                                                  double *Z, int dout)
{
    __shared__ double sL[NB][NB + 1];
    __shared__ double sInv[NB];
    for (int q = threadIdx.x; q < kb * kb; q += blockDim.x) {
        const int r = q / kb, c = q % kb;
        sL[r][c] = (c <= r) ? L[(size_t)(k0 + r) * lda + k0 + c] : 0.0;
    }
    __syncthreads();
    if (threadIdx.x < kb)
        sInv[threadIdx.x] = 1.0 / sL[threadIdx.x][threadIdx.x];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int o = warp; o < dout; o += 8) {
        double z0 = lane < kb ? Z[(size_t)(k0 + lane) * dout + o] : 0.0;
        double z1 = lane + 32 < kb ? Z[(size_t)(k0 + lane + 32) * dout + o] : 0.0;
        for (int j = 0; j < kb; ++j) {
            const double zj = __shfl_sync(kFull, j < 32 ? z0 : z1, j & 31) * sInv[j];
            if (lane == (j & 31)) {
                if (j < 32)
                    z0 = zj;
                else
                    z1 = zj;
            }
            if (lane > j && lane < kb)
                z0 = fma(-zj, sL[lane][j], z0);
            if (lane + 32 > j && lane + 32 < kb)
                z1 = fma(-zj, sL[lane + 32][j], z1);
        }
        if (lane < kb)
            Z[(size_t)(k0 + lane) * dout + o] = z0;
        if (lane + 32 < kb)
            Z[(size_t)(k0 + lane + 32) * dout + o] = z1;
    }
}

// Rows r >= k0 + kb: Z[r] -= L[r][k0:k0+kb] Z[k0:k0+kb]; one warp per row.
__global__ void __launch_bounds__(256) k_fwd_update(const double *L, int n, int lda, int k0,
                                                    int kb, double *Z, int dout)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = k0 + kb + blockIdx.x * 8 + warp;
    if (r >= n)
        return;
    const double *Lr = L + (size_t)r * lda + k0;
    const double l0 = lane < kb ? Lr[lane] : 0.0;
    const double l1 = lane + 32 < kb ? Lr[lane + 32] : 0.0;
    for (int o = 0; o < dout; ++o) {
        double v = 0.0;
        if (lane < kb)
            v = l0 * Z[(size_t)(k0 + lane) * dout + o];
        if (lane + 32 < kb)
            v = fma(l1, Z[(size_t)(k0 + lane + 32) * dout + o], v);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
            v += __shfl_xor_sync(kFull, v, off);
        if (lane == 0)
            Z[(size_t)r * dout + o] -= v;
    }
}

// Backward L^T X = Z, panels from the last one: the diagonal block (rows
// eliminated from the last, x_j = z_j / L_jj, z_r -= L_jr x_j for r < j).
__global__ void __launch_bounds__(256) k_bwd_diag(const double *L, int lda, int k0, int kb,
                                                  double *Z, int dout)
{
    __shared__ double sL[NB][NB + 1];
    __shared__ double sInv[NB];
    for (int q = threadIdx.x; q < kb * kb; q += blockDim.x) {
        const int r = q / kb, c = q % kb;
        sL[r][c] = (c <= r) ? L[(size_t)(k0 + r) * lda + k0 + c] : 0.0;
    }
    __syncthreads();
    if (threadIdx.x < kb)
        sInv[threadIdx.x] = 1.0 / sL[threadIdx.x][threadIdx.x];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int o = warp; o < dout; o += 8) {
        double z0 = lane < kb ? Z[(size_t)(k0 + lane) * dout + o] : 0.0;
        double z1 = lane + 32 < kb ? Z[(size_t)(k0 + lane + 32) * dout + o] : 0.0;
        for (int j = kb - 1; j >= 0; --j) {
            const double xj = __shfl_sync(kFull, j < 32 ? z0 : z1, j & 31) * sInv[j];
            if (lane == (j & 31)) {
                if (j < 32)
                    z0 = xj;
                else
                    z1 = xj;
            }
            if (lane < j)
                z0 = fma(-xj, sL[j][lane], z0);
            if (lane + 32 < j)
                z1 = fma(-xj, sL[j][lane + 32], z1);
        }
        if (lane < kb)
            Z[(size_t)(k0 + lane) * dout + o] = z0;
        if (lane + 32 < kb)
            Z[(size_t)(k0 + lane + 32) * dout + o] = z1;
    }
}

// Rows i < k0: Z[i] -= L[k0:k0+kb][i]^T X[k0:k0+kb]; one thread per row
// (coalesced along the rows of L).
__global__ void __launch_bounds__(256) k_bwd_update(const double *L, int lda, int k0, int kb,
                                                    double *Z, int dout)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;  // rows i < k0
    if (i >= k0)
        return;
    for (int o = 0; o < dout; ++o) {
        double v = 0.0;
        for (int c = 0; c < kb; ++c)
            v = fma(L[(size_t)(k0 + c) * lda + i], Z[(size_t)(k0 + c) * dout + o], v);
        Z[(size_t)i * dout + o] -= v;
    }
}

// ------------------------------------------------ LU with partial pivoting
// Unblocked right-looking LU, one column per step (fallback path only).
__global__ void k_lu_pivot(double *A, int n, int lda, int j, int *piv, int *info)
{
    __shared__ double bv[256];
    __shared__ int bi[256];
    double best = -1.0;
    int idx = j;
    for (int r = j + threadIdx.x; r < n; r += blockDim.x) {
        double v = fabs(A[(size_t)r * lda + j]);
        if (v > best) {
            best = v;
            idx = r;
        }
    }
    bv[threadIdx.x] = best;
    bi[threadIdx.x] = idx;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            double o = bv[threadIdx.x + s];
            int oi = bi[threadIdx.x + s];
            if (o > bv[threadIdx.x] || (o == bv[threadIdx.x] && oi < bi[threadIdx.x])) {
                bv[threadIdx.x] = o;
                bi[threadIdx.x] = oi;
            }
        }
        __syncthreads();
    }
    const int p = bi[0];
    if (threadIdx.x == 0) {
        piv[j] = p;
        if (A[(size_t)p * lda + j] == 0.0 && *info == 0)
            *info = j + 1;
    }
    if (p != j)
        for (int c = threadIdx.x; c < n; c += blockDim.x) {
            double t = A[(size_t)j * lda + c];
            A[(size_t)j * lda + c] = A[(size_t)p * lda + c];
            A[(size_t)p * lda + c] = t;
        }
}

__global__ void k_lu_update(double *A, int n, int lda, int j)
{
    const double pv = A[(size_t)j * lda + j];
    if (pv == 0.0)
        return;
    for (int r = j + 1 + blockIdx.x; r < n; r += gridDim.x) {
        const double l = A[(size_t)r * lda + j] / pv;
        __syncthreads();
        if (threadIdx.x == 0)
            A[(size_t)r * lda + j] = l;
        for (int c = j + 1 + threadIdx.x; c < n; c += blockDim.x)
            A[(size_t)r * lda + c] -= l * A[(size_t)j * lda + c];
    }
}

__global__ void k_lu_solve(const double *A, int n, int lda, const int *piv, double *Z, int dout)
{
    const int o = blockIdx.x;
    if (o >= dout)
        return;
    if (threadIdx.x == 0) {
        for (int j = 0; j < n; ++j) {
            int p = piv[j];
            if (p != j) {
                double t = Z[(size_t)j * dout + o];
                Z[(size_t)j * dout + o] = Z[(size_t)p * dout + o];
                Z[(size_t)p * dout + o] = t;
            }
        }
        for (int r = 0; r < n; ++r) {
            double v = Z[(size_t)r * dout + o];
            for (int c = 0; c < r; ++c)
                v -= A[(size_t)r * lda + c] * Z[(size_t)c * dout + o];
            Z[(size_t)r * dout + o] = v;
        }
        for (int r = n - 1; r >= 0; --r) {
            double v = Z[(size_t)r * dout + o];
            for (int c = r + 1; c < n; ++c)
                v -= A[(size_t)r * lda + c] * Z[(size_t)c * dout + o];
            Z[(size_t)r * dout + o] = v / A[(size_t)r * lda + r];
        }
    }
}

__global__ void k_axpy(double *y, const double *x, size_t cnt)
{
    size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < cnt)
        y[k] += x[k];
}

// W (n x dout) -> W_out (dout x n)
__global__ void k_transpose_w(const double *W, int n, int dout, double *W_out)
{
    size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < (size_t)n * dout) {
        int i = (int)(k / dout), o = (int)(k % dout);
        W_out[(size_t)o * n + i] = W[k];
    }
}

__global__ void k_sumsq(const double *x, size_t cnt, double *out)
{
    __shared__ double s[256];
    double a = 0.0;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < cnt;
         k += (size_t)gridDim.x * blockDim.x)
        a = fma(x[k], x[k], a);
    s[threadIdx.x] = a;
    __syncthreads();
    for (int st = 128; st; st >>= 1) {
        if (threadIdx.x < st)
            s[threadIdx.x] += s[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        atomicAdd(out, s[0]);
}

// ------------------------------------------------------------------- RLS
// Px = P x
__global__ void k_gemv_rows(const double *__restrict__ P, int n, const double *__restrict__ x,
                            double *__restrict__ y)
{
    const int r = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (r >= n)
        return;
    double s = 0.0;
    for (int c = lane; c < n; c += 32)
        s = fma(P[(size_t)r * n + c], x[c], s);
    for (int off = 16; off; off >>= 1)
        s += __shfl_xor_sync(kFull, s, off);
    if (lane == 0)
        y[r] = s;
}

// scalars: denom = lambda + x.Px ; e = target - W_out x ; k = Px / denom
__global__ void k_rls_scalars(const double *x, const double *Px, int n, double lambda,
                              const double *W_out, int dout, const double *target,
                              double *scal /* [0]=denom, [1..dout]=e */)
{
    __shared__ double red[256];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        s = fma(x[i], Px[i], s);
    red[threadIdx.x] = s;
    __syncthreads();
    for (int st = 128; st; st >>= 1) {
        if (threadIdx.x < st)
            red[threadIdx.x] += red[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        scal[0] = lambda + red[0];
    __syncthreads();
    for (int o = 0; o < dout; ++o) {
        double a = 0.0;
        for (int i = threadIdx.x; i < n; i += blockDim.x)
            a = fma(W_out[(size_t)o * n + i], x[i], a);
        red[threadIdx.x] = a;
        __syncthreads();
        for (int st = 128; st; st >>= 1) {
            if (threadIdx.x < st)
                red[threadIdx.x] += red[threadIdx.x + st];
            __syncthreads();
        }
        if (threadIdx.x == 0)
            scal[1 + o] = target[o] - red[0];
        __syncthreads();
    }
}

// W_out += e k^T ; P = (P - denom k k^T) / lambda   with k = Px / denom
__global__ void k_rls_update(double *P, int n, const double *Px, const double *scal, double lambda,
                             double *W_out, int dout)
{
    const double denom = scal[0];
    const double inv = 1.0 / denom;
    const size_t total = (size_t)n * n;
    const double sc = (lambda != 1.0) ? 1.0 / lambda : 1.0;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(q / n), c = (int)(q % n);
        const double kr = inv * Px[r], kc = inv * Px[c];
        double v = P[q] + kr * (-denom * kc);
        P[q] = (lambda != 1.0) ? sc * v : v;
    }
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < (size_t)dout * n;
         q += (size_t)gridDim.x * blockDim.x) {
        const int o = (int)(q / n), i = (int)(q % n);
        W_out[q] += (inv * Px[i]) * scal[1 + o];
    }
}

__global__ void k_diag_init(double *P, int n, double v)
{
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < (size_t)n * n;
         q += (size_t)gridDim.x * blockDim.x)
        P[q] = ((q / n) == (q % n)) ? v : 0.0;
}

// online delta rule: W_out[o][i] += (lr * (target_o - y_o)) * x_i
__global__ void k_online(double *W_out, int n, int dout, const double *x, const double *y,
                         const double *target, double lr)
{
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < (size_t)dout * n;
         q += (size_t)gridDim.x * blockDim.x) {
        const int o = (int)(q / n), i = (int)(q % n);
        const double a = lr * (target[o] - y[o]);
        W_out[q] = __dadd_rn(W_out[q], __dmul_rn(a, x[i]));
    }
}

double ms_since(std::chrono::steady_clock::time_point t)
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t)
        .count();
}

}  // namespace

// per-column dot products out[o] = sum_i X[i][o] Y[i][o] (n x dout arrays),
// one block per column, fixed-order reduction
static __global__ void k_coldot(const double *__restrict__ X, const double *__restrict__ Y, int n,
                         int dout, double *__restrict__ out)
{
    __shared__ double s[256];
    const int o = blockIdx.x;
    double a = 0.0;
    for (int i = threadIdx.x; i < n; i += 256)
        a = fma(X[(size_t)i * dout + o], Y[(size_t)i * dout + o], a);
    s[threadIdx.x] = a;
    __syncthreads();
    for (int st = 128; st; st >>= 1) {
        if ((int)threadIdx.x < st)
            s[threadIdx.x] += s[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        out[o] = s[0];
}

// Y[i][o] += c[o] X[i][o]  (xpby = 0)  or  Y[i][o] = X[i][o] + c[o] Y[i][o]  (xpby = 1)
static __global__ void k_col_update(double *__restrict__ Y, const double *__restrict__ X,
                             const double *__restrict__ c, int n, int dout, int xpby)
{
    const size_t total = (size_t)n * dout;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
         k += (size_t)gridDim.x * blockDim.x) {
        const int o = (int)(k % dout);
        Y[k] = xpby ? fma(c[o], Y[k], X[k]) : fma(c[o], X[k], Y[k]);
    }
}

// largest diagonal entry (non-negative doubles compare like their bits)
static __global__ void k_diag_max(const double *__restrict__ A, int n, unsigned long long *out)
{
    double m = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double v = A[(size_t)i * n + i];
        if (v > m)
            m = v;
    }
    for (int off = 16; off; off >>= 1) {
        const double o = __shfl_xor_sync(kFull, m, off);
        if (o > m)
            m = o;
    }
    if ((threadIdx.x & 31) == 0 && m > 0.0)
        atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// ------------------------------------------------------------ factor + solve
// Factor A (n x n) in place; returns 0 or the 1-based failing pivot.
static int cholesky_inplace(cudaStream_t s, double *A, int n, int *d_info)
{
    for (int k0 = 0; k0 < n; k0 += NB) {
        const int kb = (n - k0 < NB) ? n - k0 : NB;
        k_potrf_diag<<<1, 256, 0, s>>>(A, n, n, k0, kb, d_info);
        const int rest = n - k0 - kb;
        if (rest > 0) {
            k_trsm_panel<<<(rest + 31) / 32, 256, 0, s>>>(A, n, n, k0, kb, d_info);
            const int nt = (rest + 63) / 64;
            k_syrk_update<<<nt * (nt + 1) / 2, 256, 0, s>>>(A, n, n, k0, kb, d_info);
        }
    }
    int h = 0;
    cudaMemcpyAsync(&h, d_info, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    return h;
}

static void chol_solve(cudaStream_t s, const double *L, int n, double *Z, int dout)
{
    for (int k0 = 0; k0 < n; k0 += NB) {
        const int kb = (n - k0 < NB) ? n - k0 : NB;
        k_fwd_diag<<<1, 256, 0, s>>>(L, n, k0, kb, Z, dout);
        const int rest = n - k0 - kb;
        if (rest > 0)
            k_fwd_update<<<(rest + 7) / 8, 256, 0, s>>>(L, n, n, k0, kb, Z, dout);
    }
    const int last = ((n - 1) / NB) * NB;
    for (int k0 = last; k0 >= 0; k0 -= NB) {
        const int kb = (n - k0 < NB) ? n - k0 : NB;
        k_bwd_diag<<<1, 256, 0, s>>>(L, n, k0, kb, Z, dout);
        if (k0 > 0)
            k_bwd_update<<<(k0 + 255) / 256, 256, 0, s>>>(L, n, k0, kb, Z, dout);
    }
}

static int lu_factor_solve(cudaStream_t s, double *A, int n, int *d_piv, int *d_info, double *Z,
                           int dout)
{
    for (int j = 0; j < n; ++j) {
        k_lu_pivot<<<1, 256, 0, s>>>(A, n, n, j, d_piv, d_info);
        int rows = n - j - 1;
        if (rows > 0)
            k_lu_update<<<rows < 1024 ? rows : 1024, 256, 0, s>>>(A, n, n, j);
    }
    int h = 0;
    cudaMemcpyAsync(&h, d_info, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    if (h)
        return h;
    k_lu_solve<<<dout, 32, 0, s>>>(A, n, n, d_piv, Z, dout);
    return 0;
}

// Residual R = Phi^T (Y - Phi W) - lambda W for rows [t0, t1).
static void ridge_residual(cudaStream_t s, const double *Phi, int n, size_t t0, size_t t1,
                           const double *Y, const double *W, int dout, double lambda, double *E,
                           double *part, int parts, double *R)
{
    const size_t rows = t1 - t0;
    k_resid_rows<<<(unsigned)((rows + 7) / 8), 256, 0, s>>>(Phi, n, t0, t1, Y, W, dout, E);
    dim3 g((n + 127) / 128, parts);
    k_xt_e_part<<<g, 128, 0, s>>>(Phi, n, t0, t1, E, dout, parts, part);
    const size_t tot = (size_t)n * dout;
    k_reduce_parts<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(part, parts, n, dout, W, lambda,
                                                                 R);
}

static double device_norm(cudaStream_t s, const double *x, size_t cnt, double *d_tmp)
{
    cudaMemsetAsync(d_tmp, 0, sizeof(double), s);
    k_sumsq<<<64, 256, 0, s>>>(x, cnt, d_tmp);
    double h = 0.0;
    cudaMemcpyAsync(&h, d_tmp, sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    return sqrt(h);
}

// Dual-form ridge for T - w0 < n: K = Phi_w Phi_w^T + lambda I (FP64 Gram of
// the transposed rows), Cholesky (pivoted LU if it fails, as dgesv would),
// alpha = K^-1 Y_w, W = Phi_w^T alpha; B = Phi_w^T Y_w for the residual check.
// E (T x dout) is used as the right-hand side and holds alpha in rows w0..T-1.
static int ridge_dual(cudaStream_t s, const double *Phi, int n, size_t T, size_t w0,
                      const double *Y, int dout, double lambda, sp_ridge_report *rep, double *W,
                      double *B, double *E, double *part, int parts, int *info, int *piv)
{
    int rc = SP_OK;
    const size_t tw = T - w0;
    const int m = (int)tw;
    double *Pt = nullptr, *K = nullptr;
    const size_t tot = (size_t)n * dout;
    const dim3 gp((n + 127) / 128, parts);
    auto tg = std::chrono::steady_clock::now();
    RK(sp_cuda_malloc(&Pt, (size_t)n * tw * sizeof(double)));
    RK(sp_cuda_malloc(&K, tw * tw * sizeof(double)));
    {
        dim3 g((n + 31) / 32, (unsigned)((tw + 31) / 32));
        k_rows_to_cols<<<g, dim3(32, 8), 0, s>>>(Phi, n, w0, T, Pt);
        const int nt = (m + 63) / 64;
        k_syrk_f64<<<nt * (nt + 1) / 2, 256, 0, s>>>(Pt, m, 0, (size_t)n, K, m);
        k_add_diag<<<(m + 255) / 256, 256, 0, s>>>(K, m, m, lambda);
        k_xt_e_part<<<gp, 128, 0, s>>>(Phi, n, w0, T, Y, dout, parts, part);
        k_reduce_parts<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(part, parts, n, dout, nullptr,
                                                                     0.0, B);
        RK(cudaMemcpyAsync(E, Y, T * dout * sizeof(double), cudaMemcpyDeviceToDevice, s));
        RK(cudaStreamSynchronize(s));
        RK(cudaGetLastError());
        rep->gram_ms = ms_since(tg);
    }
    {
        auto tf = std::chrono::steady_clock::now();
        double *Z = E + w0 * dout;
        if (cholesky_inplace(s, K, m, info)) {
            rep->factor_failed = 1;
            rep->lu_fallback = 1;
            RK(cudaMemsetAsync(info, 0, sizeof(int), s));
            const int nt = (m + 63) / 64;
            k_syrk_f64<<<nt * (nt + 1) / 2, 256, 0, s>>>(Pt, m, 0, (size_t)n, K, m);
            k_add_diag<<<(m + 255) / 256, 256, 0, s>>>(K, m, m, lambda);
            if (lu_factor_solve(s, K, m, piv, info, Z, dout)) {
                rc = SP_RIDGE_SINGULAR;
                goto out;
            }
        } else {
            chol_solve(s, K, m, Z, dout);
        }
        k_xt_e_part<<<gp, 128, 0, s>>>(Phi, n, w0, T, E, dout, parts, part);
        k_reduce_parts<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(part, parts, n, dout, nullptr,
                                                                     0.0, W);
        RK(cudaStreamSynchronize(s));
        RK(cudaGetLastError());
        rep->factor_ms = ms_since(tf);
    }
out:
    cudaStreamSynchronize(s);
    if (Pt)
        sp_cuda_free(Pt);
    if (K)
        sp_cuda_free(K);
    return rc;
}

// Mixed-precision solve of (Phi_w^T Phi_w + lambda I) W = B given A = G + lambda I
// with G the split tensor-core Gram. The rounding error of G can exceed
// lambda, so A itself may be indefinite: the preconditioner is the FP64
// Cholesky factor of A + delta I, delta = eps * max diag (raised tenfold until
// the factorisation succeeds), and the system is solved by preconditioned
// conjugate gradients per output column whose operator p -> Phi^T (Phi p) +
// lambda p is applied in FP64 from the states themselves. So the answer is
// the FP64 ridge solution to the stated residual; the Gram's precision only
// sets how many iterations that takes.
static int ridge_mixed(cudaStream_t s, const double *Phi, int n, size_t T, size_t w0,
                       const double *Y, int dout, double lambda, int mode,
                       const sp_ridge_opts *o, sp_ridge_report *rep, double *A, double *B,
                       double *W, double *R, double *E, double *part, int parts, double *tmp,
                       int *info)
{
    int rc = SP_OK;
    const size_t nn = (size_t)n * n, tot = (size_t)n * dout;
    const unsigned gb = (unsigned)((tot + 255) / 256 < 4096 ? (tot + 255) / 256 : 4096);
    double *A0 = nullptr, *Z = nullptr, *P = nullptr, *Q = nullptr, *Yz = nullptr, *c = nullptr,
           *dots = nullptr;
    double h_rz[16], h_pq[16], h_c[16];
    auto tf = std::chrono::steady_clock::now();
    RK(sp_cuda_malloc(&A0, nn * sizeof(double)));
    RK(sp_cuda_malloc(&Z, tot * sizeof(double)));
    RK(sp_cuda_malloc(&P, tot * sizeof(double)));
    RK(sp_cuda_malloc(&Q, tot * sizeof(double)));
    RK(sp_cuda_malloc(&Yz, (T ? T : 1) * (size_t)dout * sizeof(double)));
    RK(sp_cuda_malloc(&c, 16 * sizeof(double)));
    RK(sp_cuda_malloc(&dots, 16 * sizeof(double)));
    RK(cudaMemsetAsync(Yz, 0, (T ? T : 1) * (size_t)dout * sizeof(double), s));
    RK(cudaMemcpyAsync(A0, A, nn * sizeof(double), cudaMemcpyDeviceToDevice, s));
    {
        RK(cudaMemsetAsync(tmp, 0, sizeof(double), s));
        k_diag_max<<<(n + 255) / 256, 256, 0, s>>>(A, n, (unsigned long long *)tmp);
        double dmax = 0.0;
        RK(cudaMemcpyAsync(&dmax, tmp, sizeof(double), cudaMemcpyDeviceToHost, s));
        RK(cudaStreamSynchronize(s));
        double delta = (mode == 1 ? 1e-4 : 1e-5) * dmax;
        int ok = 0;
        for (int attempt = 0; attempt < 6 && !ok; ++attempt, delta *= 10.0) {
            if (attempt > 0) {
                rep->factor_failed = 1;
                RK(cudaMemcpyAsync(A, A0, nn * sizeof(double), cudaMemcpyDeviceToDevice, s));
                RK(cudaMemsetAsync(info, 0, sizeof(int), s));
            }
            k_add_diag<<<(n + 255) / 256, 256, 0, s>>>(A, n, n, delta);
            ok = cholesky_inplace(s, A, n, info) == 0;
        }
        if (!ok) {
            rc = SP_RIDGE_SINGULAR;
            goto out;
        }
        rep->factor_ms = ms_since(tf);
    }
    {
        auto tr = std::chrono::steady_clock::now();
        const double bnorm = device_norm(s, B, tot, tmp);
        const double bden = bnorm > 0 ? bnorm : 1.0;
        // W = M^-1 B, R = B - A W (FP64 from Phi), Z = M^-1 R, P = Z
        RK(cudaMemcpyAsync(W, B, tot * sizeof(double), cudaMemcpyDeviceToDevice, s));
        chol_solve(s, A, n, W, dout);
        ridge_residual(s, Phi, n, w0, T, Y, W, dout, lambda, E, part, parts, R);
        RK(cudaMemcpyAsync(Z, R, tot * sizeof(double), cudaMemcpyDeviceToDevice, s));
        chol_solve(s, A, n, Z, dout);
        RK(cudaMemcpyAsync(P, Z, tot * sizeof(double), cudaMemcpyDeviceToDevice, s));
        k_coldot<<<dout, 256, 0, s>>>(R, Z, n, dout, dots);
        RK(cudaMemcpyAsync(h_rz, dots, dout * sizeof(double), cudaMemcpyDeviceToHost, s));
        int it = 0;
        double rel = device_norm(s, R, tot, tmp) / bden;
        while (rel > o->refine_tol && it < o->max_refine) {
            // Q = -(A P): the residual form with zero targets
            ridge_residual(s, Phi, n, w0, T, Yz, P, dout, lambda, E, part, parts, Q);
            k_coldot<<<dout, 256, 0, s>>>(P, Q, n, dout, dots);
            RK(cudaMemcpyAsync(h_pq, dots, dout * sizeof(double), cudaMemcpyDeviceToHost, s));
            RK(cudaStreamSynchronize(s));
            for (int k = 0; k < dout; ++k)
                h_c[k] = (h_pq[k] != 0.0) ? h_rz[k] / -h_pq[k] : 0.0;  // alpha
            RK(cudaMemcpyAsync(c, h_c, dout * sizeof(double), cudaMemcpyHostToDevice, s));
            k_col_update<<<gb, 256, 0, s>>>(W, P, c, n, dout, 0);  // W += alpha P
            k_col_update<<<gb, 256, 0, s>>>(R, Q, c, n, dout, 0);  // R -= alpha A P
            RK(cudaMemcpyAsync(Z, R, tot * sizeof(double), cudaMemcpyDeviceToDevice, s));
            chol_solve(s, A, n, Z, dout);
            k_coldot<<<dout, 256, 0, s>>>(R, Z, n, dout, dots);
            double h_rz2[16];
            RK(cudaMemcpyAsync(h_rz2, dots, dout * sizeof(double), cudaMemcpyDeviceToHost, s));
            RK(cudaStreamSynchronize(s));
            for (int k = 0; k < dout; ++k) {
                h_c[k] = (h_rz[k] != 0.0) ? h_rz2[k] / h_rz[k] : 0.0;  // beta
                h_rz[k] = h_rz2[k];
            }
            RK(cudaMemcpyAsync(c, h_c, dout * sizeof(double), cudaMemcpyHostToDevice, s));
            k_col_update<<<gb, 256, 0, s>>>(P, Z, c, n, dout, 1);  // P = Z + beta P
            ++it;
            rel = device_norm(s, R, tot, tmp) / bden;
        }
        // the reported residual is recomputed from Phi, not the recurrence
        ridge_residual(s, Phi, n, w0, T, Y, W, dout, lambda, E, part, parts, R);
        rep->rel_residual = device_norm(s, R, tot, tmp) / bden;
        rep->refine_iters = it;
        rep->refine_ms = ms_since(tr);
        RK(cudaGetLastError());
    }
out:
    cudaStreamSynchronize(s);
    void *bufs[] = {A0, Z, P, Q, Yz, c, dots};
    for (void *b : bufs)
        if (b)
            sp_cuda_free(b);
    return rc;
}

// Work buffers of the primal solve, kept across calls by a caller that fits
// many readouts in a row (the batched fits): grown to the largest sizes seen,
// freed by sp_ridge_ws_free.
struct sp_ridge_ws {
    double *A = nullptr, *B = nullptr, *W = nullptr, *R = nullptr, *E = nullptr,
           *part = nullptr, *tmp = nullptr;
    int *info = nullptr, *piv = nullptr;
    size_t cap_nn = 0, cap_nd = 0, cap_td = 0, cap_n = 0;
};

extern "C" sp_ridge_ws *sp_ridge_ws_new(void) { return new sp_ridge_ws(); }

static void ws_release(sp_ridge_ws *w)
{
    void *bufs[] = {w->A, w->B, w->W, w->R, w->E, w->part, w->tmp, w->info, w->piv};
    for (void *b : bufs)
        if (b)
            sp_cuda_free(b);
    *w = sp_ridge_ws();
}

extern "C" void sp_ridge_ws_free(sp_ridge_ws *w)
{
    if (!w)
        return;
    ws_release(w);
    delete w;
}

// Buffers for n neurons, T rows and dout (<= 16) outputs, reusing what is
// large enough. The caller's stream must be idle (the batched fits wait for
// each instance before the next).
static int ws_ensure(sp_ridge_ws *w, int n, size_t T, int dout, int parts)
{
    const size_t nn = (size_t)n * n, nd = (size_t)n * dout, td = (T ? T : 1) * (size_t)dout;
    if (nn <= w->cap_nn && nd <= w->cap_nd && td <= w->cap_td && (size_t)n <= w->cap_n)
        return SP_OK;
    const size_t cnn = nn > w->cap_nn ? nn : w->cap_nn, cnd = nd > w->cap_nd ? nd : w->cap_nd,
                 ctd = td > w->cap_td ? td : w->cap_td,
                 cn = (size_t)n > w->cap_n ? (size_t)n : w->cap_n;
    ws_release(w);
    int rc = SP_OK;
    RK(sp_cuda_malloc(&w->A, cnn * sizeof(double)));
    RK(sp_cuda_malloc(&w->B, cnd * sizeof(double)));
    RK(sp_cuda_malloc(&w->W, cnd * sizeof(double)));
    RK(sp_cuda_malloc(&w->R, cnd * sizeof(double)));
    RK(sp_cuda_malloc(&w->E, ctd * sizeof(double)));
    RK(sp_cuda_malloc(&w->part, (size_t)parts * cnd * sizeof(double)));
    RK(sp_cuda_malloc(&w->tmp, 4 * sizeof(double)));
    RK(sp_cuda_malloc(&w->info, sizeof(int)));
    RK(sp_cuda_malloc(&w->piv, cn * sizeof(int)));
    w->cap_nn = cnn;
    w->cap_nd = cnd;
    w->cap_td = ctd;
    w->cap_n = cn;
    return SP_OK;
out:
    ws_release(w);
    return rc;
}

// One group of at most 16 outputs of sp_ridge_phi (below). Work buffers come
// from `ws` when given, else are allocated for the call.
static int ridge_phi_group(cudaStream_t s, const double *Phi, int n, size_t T,
                           const double *Y, int dout, double lambda, const sp_ridge_opts *o,
                           sp_ridge_report *rep, double *d_W_out, sp_ridge_ws *ws)
{
    int rc = SP_OK;
    double *A = nullptr, *Aw = nullptr, *B = nullptr, *W = nullptr, *R = nullptr, *E = nullptr,
           *part = nullptr, *tmp = nullptr;
    int *info = nullptr, *piv = nullptr;
    const int parts = 64;
    const size_t w0 = o->washout;
    if (dout == 0)
        return SP_OK;
    if (dout > 16)
        return SP_EINVAL; /* per-thread accumulators below hold up to 16 outputs */
    if (ws) {
        rc = ws_ensure(ws, n, T, dout, parts);
        if (rc)
            return rc;
        A = ws->A;
        B = ws->B;
        W = ws->W;
        R = ws->R;
        E = ws->E;
        part = ws->part;
        tmp = ws->tmp;
        info = ws->info;
        piv = ws->piv;
    } else {
        RK(sp_cuda_malloc(&A, (size_t)n * n * sizeof(double)));
        RK(sp_cuda_malloc(&B, (size_t)n * dout * sizeof(double)));
        RK(sp_cuda_malloc(&W, (size_t)n * dout * sizeof(double)));
        RK(sp_cuda_malloc(&R, (size_t)n * dout * sizeof(double)));
        RK(sp_cuda_malloc(&E, (T ? T : 1) * (size_t)dout * sizeof(double)));
        RK(sp_cuda_malloc(&part, (size_t)parts * n * dout * sizeof(double)));
        RK(sp_cuda_malloc(&tmp, 4 * sizeof(double)));
        RK(sp_cuda_malloc(&info, sizeof(int)));
        RK(sp_cuda_malloc(&piv, (size_t)n * sizeof(int)));
    }
    RK(cudaMemsetAsync(info, 0, sizeof(int), s));

    if (lambda > 0.0 && 2 * (T - w0) <= (size_t)n) {
        // Fewer fitted rows than half the neurons: the dual form
        // W = Phi_w^T (Phi_w Phi_w^T + lambda I)^-1 Y_w, algebraically the same
        // solution, factors a (T - w0)^2 matrix instead of n^2. (lambda = 0
        // keeps the primal system, singular here, so that the call fails and
        // leaves W_out as the reference's dgesv does.)
        rc = ridge_dual(s, Phi, n, T, w0, Y, dout, lambda, rep, W, B, E, part, parts, info, piv);
        if (rc)
            goto out;
        rep->dual = 1;
        rep->gram_mode_used = 0;
        const double bnorm = device_norm(s, B, (size_t)n * dout, tmp);
        ridge_residual(s, Phi, n, w0, T, Y, W, dout, lambda, E, part, parts, R);
        rep->rel_residual = device_norm(s, R, (size_t)n * dout, tmp) / (bnorm > 0 ? bnorm : 1.0);
        rep->refine_iters = 0;
        const size_t tot = (size_t)n * dout;
        k_transpose_w<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(W, n, dout, d_W_out);
        RK(cudaStreamSynchronize(s));
        RK(cudaGetLastError());
        goto out;
    }

    {
        auto tg = std::chrono::steady_clock::now();
        int mode = o->gram_mode;
        const int slices = o->gram_slices > 0 ? o->gram_slices : SP_GRAM_INT8_SLICES;
        if ((mode == SP_GRAM_BF16X3 || mode == SP_GRAM_TF32X3 || mode == SP_GRAM_INT8) &&
            sp_gram_tc_available()) {
            rc = sp_gram_tc(s, mode, slices, Phi, n, w0, T, A, n);
            if (rc == SP_EINVAL && mode == SP_GRAM_INT8) {
                // a state that is not finite: the FP64 Gram, as the reference
                rc = SP_OK;
                mode = 0;
                const int nt = (n + 63) / 64;
                k_syrk_f64<<<nt * (nt + 1) / 2, 256, 0, s>>>(Phi, n, w0, T, A, n);
            }
            if (rc)
                goto out;
        } else {
            mode = 0;
            const int nt = (n + 63) / 64;
            k_syrk_f64<<<nt * (nt + 1) / 2, 256, 0, s>>>(Phi, n, w0, T, A, n);
        }
        rep->gram_mode_used = mode;
        dim3 g((n + 127) / 128, parts);
        k_xt_e_part<<<g, 128, 0, s>>>(Phi, n, w0, T, Y, dout, parts, part);
        const size_t tot = (size_t)n * dout;
        k_reduce_parts<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(part, parts, n, dout, nullptr,
                                                                     0.0, B);
        k_add_diag<<<(n + 255) / 256, 256, 0, s>>>(A, n, n, lambda);
        RK(cudaStreamSynchronize(s));
        RK(cudaGetLastError());
        rep->gram_ms = ms_since(tg);
    }

    if (rep->gram_mode_used == SP_GRAM_BF16X3 || rep->gram_mode_used == SP_GRAM_TF32X3) {
        // an FP32-accumulated Gram is too coarse to factor directly at small
        // lambda: Cholesky-preconditioned CG on the FP64 operator
        rc = ridge_mixed(s, Phi, n, T, w0, Y, dout, lambda, rep->gram_mode_used, o, rep, A, B, W,
                         R, E, part, parts, tmp, info);
        if (rc)
            goto out;
        const size_t tot = (size_t)n * dout;
        k_transpose_w<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(W, n, dout, d_W_out);
        RK(cudaStreamSynchronize(s));
        RK(cudaGetLastError());
        goto out;
    }

    {
        auto tf = std::chrono::steady_clock::now();
        RK(cudaMemcpyAsync(W, B, (size_t)n * dout * sizeof(double), cudaMemcpyDeviceToDevice, s));
        int bad = cholesky_inplace(s, A, n, info);
        if (bad) {
            // dgesv semantics: LU with partial pivoting on the original matrix
            rep->factor_failed = 1;
            rep->lu_fallback = 1;
            RK(cudaMemsetAsync(info, 0, sizeof(int), s));
            if (rep->gram_mode_used != 0) {
                rc = sp_gram_tc(s, rep->gram_mode_used,
                                o->gram_slices > 0 ? o->gram_slices : SP_GRAM_INT8_SLICES, Phi,
                                n, w0, T, A, n);
                if (rc)
                    goto out;
            } else {
                const int nt = (n + 63) / 64;
                k_syrk_f64<<<nt * (nt + 1) / 2, 256, 0, s>>>(Phi, n, w0, T, A, n);
            }
            k_add_diag<<<(n + 255) / 256, 256, 0, s>>>(A, n, n, lambda);
            int lbad = lu_factor_solve(s, A, n, piv, info, W, dout);
            if (lbad) {
                rc = SP_RIDGE_SINGULAR;
                goto out;
            }
            rep->factor_ms = ms_since(tf);
        } else {
            // cholesky_inplace has waited for the factorisation
            rep->factor_ms = ms_since(tf);
            auto ts = std::chrono::steady_clock::now();
            chol_solve(s, A, n, W, dout);
            RK(cudaStreamSynchronize(s));
            rep->solve_ms = ms_since(ts);
        }
        RK(cudaStreamSynchronize(s));
        RK(cudaGetLastError());
    }

    {
        // iterative refinement with FP64 residuals from Phi itself
        auto tr = std::chrono::steady_clock::now();
        const double bnorm = device_norm(s, B, (size_t)n * dout, tmp);
        int it = 0;
        double rel = 0.0;
        const int maxit = rep->lu_fallback ? 0 : o->max_refine;
        for (;;) {
            ridge_residual(s, Phi, n, w0, T, Y, W, dout, lambda, E, part, parts, R);
            rel = device_norm(s, R, (size_t)n * dout, tmp) / (bnorm > 0 ? bnorm : 1.0);
            if (rel <= o->refine_tol || it >= maxit)
                break;
            chol_solve(s, A, n, R, dout);
            const size_t tot = (size_t)n * dout;
            k_axpy<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(W, R, tot);
            ++it;
        }
        rep->refine_iters = it;
        rep->rel_residual = rel;
        rep->refine_ms = ms_since(tr);
    }

    {
        const size_t tot = (size_t)n * dout;
        // W (n x dout) -> W_out (dout x n)
        k_transpose_w<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(W, n, dout, d_W_out);
        RK(cudaStreamSynchronize(s));
        RK(cudaGetLastError());
    }
out:
    cudaStreamSynchronize(s);
    if (!ws) {
        void *bufs[] = {A, Aw, B, W, R, E, part, tmp, info, piv};
        for (void *b : bufs)
            if (b)
                sp_cuda_free(b);
    } else if (Aw) {
        sp_cuda_free(Aw);
    }
    return rc;
}

extern "C" int sp_gram_fp64(cudaStream_t s, const double *X, int n, size_t t0, size_t t1,
                            double *C, int ldc)
{
    const int nt = (n + 63) / 64;
    k_syrk_f64<<<nt * (nt + 1) / 2, 256, 0, s>>>(X, n, t0, t1, C, ldc);
    return cudaGetLastError() == cudaSuccess ? SP_OK : SP_EINTERNAL;
}

// Ridge on states already on the device: Phi [T x n] row-major (neuron order),
// Y [T x dout]; rows [washout, T) enter the Gram. On success d_W_out [dout x n]
// holds the solution; SP_RIDGE_SINGULAR leaves it untouched (dgesv failure in
// the reference leaves W_out as it was). The solver's per-thread accumulators
// hold 16 outputs; with more, the outputs are solved 16 at a time -- the system
// matrix is the same for all of them -- each group's targets copied to a
// contiguous block and its rows of W gathered in a work array that reaches
// d_W_out only when every group has succeeded.
extern "C" int sp_ridge_phi(cudaStream_t s, const double *Phi, int n, size_t T,
                            const double *Y, int dout, double lambda, const sp_ridge_opts *o,
                            sp_ridge_report *rep, double *d_W_out);

extern "C" int sp_ridge_phi_ws(cudaStream_t s, const double *Phi, int n, size_t T,
                               const double *Y, int dout, double lambda, const sp_ridge_opts *o,
                               sp_ridge_report *rep, double *d_W_out, sp_ridge_ws *ws)
{
    if (dout <= 16)
        return ridge_phi_group(s, Phi, n, T, Y, dout, lambda, o, rep, d_W_out, ws);
    return sp_ridge_phi(s, Phi, n, T, Y, dout, lambda, o, rep, d_W_out);
}

extern "C" int sp_ridge_phi(cudaStream_t s, const double *Phi, int n, size_t T,
                            const double *Y, int dout, double lambda, const sp_ridge_opts *o,
                            sp_ridge_report *rep, double *d_W_out)
{
    if (dout <= 16)
        return ridge_phi_group(s, Phi, n, T, Y, dout, lambda, o, rep, d_W_out, nullptr);
    int rc = SP_OK;
    double *Yg = nullptr, *Wall = nullptr;
    sp_ridge_report sum;
    memset(&sum, 0, sizeof(sum));
    RK(sp_cuda_malloc(&Yg, (T ? T : 1) * 16 * sizeof(double)));
    RK(sp_cuda_malloc(&Wall, (size_t)dout * n * sizeof(double)));
    for (int g0 = 0; g0 < dout && !rc; g0 += 16) {
        const int dg = dout - g0 < 16 ? dout - g0 : 16;
        if (T)
            RK(cudaMemcpy2DAsync(Yg, (size_t)dg * sizeof(double), Y + g0,
                                 (size_t)dout * sizeof(double), (size_t)dg * sizeof(double), T,
                                 cudaMemcpyDeviceToDevice, s));
        sp_ridge_report r1;
        memset(&r1, 0, sizeof(r1));
        rc = ridge_phi_group(s, Phi, n, T, Yg, dg, lambda, o, &r1, Wall + (size_t)g0 * n,
                             nullptr);
        sum.gram_mode_used = r1.gram_mode_used;
        sum.dual = r1.dual;
        sum.refine_iters = r1.refine_iters > sum.refine_iters ? r1.refine_iters : sum.refine_iters;
        sum.rel_residual = r1.rel_residual > sum.rel_residual ? r1.rel_residual : sum.rel_residual;
        sum.gram_ms += r1.gram_ms;
        sum.factor_ms += r1.factor_ms;
        sum.solve_ms += r1.solve_ms;
        sum.refine_ms += r1.refine_ms;
        sum.factor_failed |= r1.factor_failed;
        sum.lu_fallback |= r1.lu_fallback;
    }
    if (!rc)
        RK(cudaMemcpyAsync(d_W_out, Wall, (size_t)dout * n * sizeof(double),
                           cudaMemcpyDeviceToDevice, s));
out:
    cudaStreamSynchronize(s);
    if (Yg)
        sp_cuda_free(Yg);
    if (Wall)
        sp_cuda_free(Wall);
    sum.collect_ms = rep->collect_ms;
    *rep = sum;
    return rc;
}

// Ridge on caller-provided states (host arrays): Phi [T x n], Y [T x dout];
// writes W_out [dout x n] to the host. Same solver (and dual/split choices) as
// the reservoir readouts, on the current device and a stream of its own.
extern "C" int sp_ridge_host(const double *h_phi, size_t T, int n, const double *h_y, int dout,
                             double lambda, const sp_ridge_opts *o, sp_ridge_report *rep,
                             double *h_w_out)
{
    int rc = SP_OK;
    cudaStream_t s = nullptr;
    double *Phi = nullptr, *Y = nullptr, *Wt = nullptr;
    memset(rep, 0, sizeof(*rep));
    if (dout <= 0 || n <= 0 || T == 0 || o->washout >= T)
        return SP_EINVAL;
    auto t0 = std::chrono::steady_clock::now();
    RK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    RK(sp_cuda_malloc(&Phi, T * (size_t)n * sizeof(double)));
    RK(sp_cuda_malloc(&Y, T * (size_t)dout * sizeof(double)));
    RK(sp_cuda_malloc(&Wt, (size_t)n * dout * sizeof(double)));
    RK(cudaMemcpyAsync(Phi, h_phi, T * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s));
    RK(cudaMemcpyAsync(Y, h_y, T * (size_t)dout * sizeof(double), cudaMemcpyHostToDevice, s));
    RK(cudaStreamSynchronize(s));
    rep->collect_ms = ms_since(t0);
    rc = sp_ridge_phi(s, Phi, n, T, Y, dout, lambda, o, rep, Wt);
    if (rc)
        goto out;
    RK(cudaMemcpyAsync(h_w_out, Wt, (size_t)n * dout * sizeof(double), cudaMemcpyDeviceToHost, s));
    RK(cudaStreamSynchronize(s));
out:
    if (s)
        cudaStreamSynchronize(s);
    void *bufs[] = {Phi, Y, Wt};
    for (void *b : bufs)
        if (b)
            sp_cuda_free(b);
    if (s)
        cudaStreamDestroy(s);
    return rc;
}

extern "C" int sp_dev_train_ridge(sp_dev *d, const sp_host_model *m, const double *h_u,
                                  const double *h_y, size_t T, double lambda,
                                  const sp_ridge_opts *o, sp_ridge_report *rep, double *h_W_out)
{
    int rc = SP_OK;
    const int n = d->n, dout = d->dout;
    cudaStream_t s = d->stream;
    double *Phi = nullptr, *Y = nullptr, *Wt = nullptr;
    memset(rep, 0, sizeof(*rep));
    if (dout == 0)
        return SP_OK;
    auto tstart = std::chrono::steady_clock::now();

    rc = sp_dev_reset_neurons(d, m);
    if (rc)
        return rc;
    RK(sp_cuda_malloc(&Phi, (T ? T : 1) * (size_t)n * sizeof(double)));
    RK(sp_cuda_malloc(&Y, (T ? T : 1) * (size_t)dout * sizeof(double)));
    RK(sp_cuda_malloc(&Wt, (size_t)n * dout * sizeof(double)));
    RK(cudaMemcpyAsync(Y, h_y, T * dout * sizeof(double), cudaMemcpyHostToDevice, s));
    {
        sp_run_args a;
        memset(&a, 0, sizeof(a));
        a.u = h_u;
        a.T = T;
        a.d_phi = Phi;
        a.sync = 1;
        rc = sp_dev_run(d, &a);
        if (rc)
            goto out;
    }
    rep->collect_ms = ms_since(tstart);
    rc = sp_ridge_phi(s, Phi, n, T, Y, dout, lambda, o, rep, Wt);
    if (rc == SP_RIDGE_SINGULAR) {
        // singular: the reference leaves W_out unchanged and warns
        fprintf(stderr, "Warning: Ridge regression failed (singular system).\n");
        rc = SP_OK;
        goto out;
    }
    if (rc)
        goto out;
    RK(cudaMemcpyAsync(h_W_out, Wt, (size_t)n * dout * sizeof(double), cudaMemcpyDeviceToHost, s));
    rc = sp_dev_w_out_from_nat(d, Wt);
    if (rc)
        goto out;
    RK(cudaStreamSynchronize(s));
    RK(cudaGetLastError());
out:
    cudaStreamSynchronize(s);
    void *bufs[] = {Phi, Y, Wt};
    for (void *b : bufs)
        if (b)
            sp_cuda_free(b);
    return rc;
}

extern "C" int sp_dev_train_rls(sp_dev *d, const sp_host_model *m, const double *h_u,
                                const double *h_y, size_t T, double delta, double lambda,
                                double *h_W_out)
{
    // state, W_out and P live in position space (holes keep x = 0 and stay inert)
    int rc = SP_OK;
    const int rs = d->rs, n = d->n, dout = d->dout;
    cudaStream_t s = d->stream;
    double *P = nullptr, *Px = nullptr, *scal = nullptr, *Yd = nullptr, *Wn = nullptr;
    RK(sp_cuda_malloc(&P, (size_t)rs * rs * sizeof(double)));
    RK(sp_cuda_malloc(&Px, (size_t)rs * sizeof(double)));
    RK(sp_cuda_malloc(&scal, (size_t)(dout + 1) * sizeof(double)));
    RK(sp_cuda_malloc(&Yd, (T ? T : 1) * (size_t)(dout ? dout : 1) * sizeof(double)));
    RK(sp_cuda_malloc(&Wn, (size_t)(dout ? dout : 1) * n * sizeof(double)));
    k_diag_init<<<1024, 256, 0, s>>>(P, rs, 1.0 / delta);
    RK(cudaMemsetAsync(d->W_out, 0, (size_t)rs * dout * sizeof(double), s));
    if (T && dout)
        RK(cudaMemcpyAsync(Yd, h_y, T * dout * sizeof(double), cudaMemcpyHostToDevice, s));
    rc = sp_dev_reset_neurons(d, m);
    if (rc)
        goto out;
    for (size_t t = 0; t < T; ++t) {
        sp_run_args a;
        memset(&a, 0, sizeof(a));
        a.u = h_u ? h_u + t * d->din : nullptr;
        a.T = 1;
        rc = sp_dev_run(d, &a);
        if (rc)
            goto out;
        k_gemv_rows<<<(rs + 7) / 8, 256, 0, s>>>(P, rs, d->V, Px);
        k_rls_scalars<<<1, 256, 0, s>>>(d->V, Px, rs, lambda, d->W_out, dout, Yd + t * dout,
                                        scal);
        k_rls_update<<<4 * d->num_sms, 256, 0, s>>>(P, rs, Px, scal, lambda, d->W_out, dout);
    }
    rc = sp_dev_w_out_to_nat(d, Wn);
    if (rc)
        goto out;
    RK(cudaMemcpyAsync(h_W_out, Wn, (size_t)n * dout * sizeof(double), cudaMemcpyDeviceToHost,
                       s));
    RK(cudaStreamSynchronize(s));
    RK(cudaGetLastError());
out:
    cudaStreamSynchronize(s);
    if (P) sp_cuda_free(P);
    if (Px) sp_cuda_free(Px);
    if (scal) sp_cuda_free(scal);
    if (Yd) sp_cuda_free(Yd);
    if (Wn) sp_cuda_free(Wn);
    return rc;
}

extern "C" int sp_dev_train_online(sp_dev *d, const double *h_target, double lr, double *h_W_out)
{
    int rc = SP_OK;
    const int rs = d->rs, n = d->n, dout = d->dout;
    cudaStream_t s = d->stream;
    double *Wn = nullptr;
    if (dout == 0)
        return SP_OK;
    // prediction with the same readout kernel as spires_compute_output
    rc = sp_dev_readout(d, d->V, 1, d->d_y);
    if (rc)
        return rc;
    RK(sp_cuda_malloc(&Wn, (size_t)dout * n * sizeof(double)));
    RK(cudaMemcpyAsync(d->d_y + dout, h_target, (size_t)dout * sizeof(double),
                       cudaMemcpyHostToDevice, s));
    k_online<<<(unsigned)(((size_t)rs * dout + 255) / 256), 256, 0, s>>>(d->W_out, rs, dout, d->V,
                                                                        d->d_y, d->d_y + dout, lr);
    rc = sp_dev_w_out_to_nat(d, Wn);
    if (rc)
        goto out;
    RK(cudaMemcpyAsync(h_W_out, Wn, (size_t)n * dout * sizeof(double), cudaMemcpyDeviceToHost,
                       s));
    RK(cudaStreamSynchronize(s));
    RK(cudaGetLastError());
out:
    cudaStreamSynchronize(s);
    if (Wn)
        sp_cuda_free(Wn);
    return rc;
}

// ---------------------------------------------------- allocation-free solve
// Ridge readout from states the caller already holds in device memory, for
// callers that cannot allocate device memory themselves: a host framework
// that owns every device buffer through its own allocator or quota, or a
// control loop that cannot afford the implicit device-wide synchronisation of
// cudaMalloc/cudaFree. All working memory is the file-scope array below,
// sized for at most SP_NA_MAX_N neurons, SP_NA_MAX_DOUT outputs and
// SP_NA_MAX_T rows (8.6 MB); every GPU that loads this library holds it until
// the process exits. The same kernels as spires_ext_train_ridge with the FP64
// Gram run in the same order, so the two agree given the same states.
#define SP_NA_MAX_N 512
#define SP_NA_MAX_DOUT 16
#define SP_NA_MAX_T 16384
#define SP_NA_PARTS 64
#define SP_NA_DOUBLES                                                                  \
    ((size_t)SP_NA_MAX_N * SP_NA_MAX_N + 3 * (size_t)SP_NA_MAX_N * SP_NA_MAX_DOUT +    \
     (size_t)SP_NA_MAX_T * SP_NA_MAX_DOUT +                                            \
     (size_t)SP_NA_PARTS * SP_NA_MAX_N * SP_NA_MAX_DOUT + 8)

static __device__ __align__(256) double g_na_scratch[SP_NA_DOUBLES];
static __device__ __align__(256) int g_na_iscratch[SP_NA_MAX_N + 8];

// Device addresses of the two arrays, looked up once per device (with that
// device current) on the first call made on it.
static double *g_na_dptr[64];
static int *g_na_iptr[64];

static int na_setup(int dev)
{
    if (dev < 0 || dev >= 64)
        return SP_EINTERNAL;
    if (g_na_dptr[dev] && g_na_iptr[dev])
        return SP_OK;
    void *pd = nullptr, *pi = nullptr;
    if (cudaGetSymbolAddress(&pd, g_na_scratch) != cudaSuccess || !pd)
        return SP_EINTERNAL;
    if (cudaGetSymbolAddress(&pi, g_na_iscratch) != cudaSuccess || !pi)
        return SP_EINTERNAL;
    g_na_dptr[dev] = (double *)pd;
    g_na_iptr[dev] = (int *)pi;
    return SP_OK;
}

extern "C" __attribute__((visibility("default"))) int
spires_ext_ridge_solve_noalloc(const double *d_states, const double *d_targets, size_t T,
                               size_t n_, size_t dout_, size_t washout, double lambda,
                               double *d_w_out, void *stream)
{
    if (!d_states || !d_targets || !d_w_out || T == 0 || n_ == 0 || dout_ == 0 || washout >= T)
        return SP_EINVAL;
    if (n_ > SP_NA_MAX_N || dout_ > SP_NA_MAX_DOUT || T > SP_NA_MAX_T) {
        fprintf(stderr,
                "spires_ext_ridge_solve_noalloc: size beyond the fixed work area "
                "(N=%zu > %d, outputs=%zu > %d or rows=%zu > %d)\n",
                n_, SP_NA_MAX_N, dout_, SP_NA_MAX_DOUT, T, SP_NA_MAX_T);
        return SP_EINVAL;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
        return SP_EINTERNAL;
    int rc = na_setup(dev);
    if (rc)
        return rc;
    const int n = (int)n_, dout = (int)dout_;
    cudaStream_t s = (cudaStream_t)stream;
    double *A = g_na_dptr[dev];
    double *B = A + (size_t)SP_NA_MAX_N * SP_NA_MAX_N;
    double *W = B + (size_t)SP_NA_MAX_N * SP_NA_MAX_DOUT;
    double *R = W + (size_t)SP_NA_MAX_N * SP_NA_MAX_DOUT;
    double *E = R + (size_t)SP_NA_MAX_N * SP_NA_MAX_DOUT;
    double *part = E + (size_t)SP_NA_MAX_T * SP_NA_MAX_DOUT;
    double *tmp = part + (size_t)SP_NA_PARTS * SP_NA_MAX_N * SP_NA_MAX_DOUT;
    int *info = g_na_iptr[dev];
    int *piv = info + 8;
    const int parts = SP_NA_PARTS;
    const size_t tot = (size_t)n * dout;
    const int maxit = 30;
    const double tol = 1e-13;

    // the work area keeps the previous call's contents: clear the flag that
    // must start at zero; every other region is fully rewritten below
    if (cudaMemsetAsync(info, 0, sizeof(int), s) != cudaSuccess)
        return SP_EINTERNAL;
    const int nt = (n + 63) / 64;
    k_syrk_f64<<<nt * (nt + 1) / 2, 256, 0, s>>>(d_states, n, washout, T, A, n);
    {
        dim3 g((n + 127) / 128, parts);
        k_xt_e_part<<<g, 128, 0, s>>>(d_states, n, washout, T, d_targets, dout, parts, part);
        k_reduce_parts<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(part, parts, n, dout,
                                                                     nullptr, 0.0, B);
    }
    k_add_diag<<<(n + 255) / 256, 256, 0, s>>>(A, n, n, lambda);
    if (cudaMemcpyAsync(W, B, tot * sizeof(double), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
        return SP_EINTERNAL;
    int bad = cholesky_inplace(s, A, n, info);
    bool lu = false;
    if (bad) {
        lu = true;
        cudaMemsetAsync(info, 0, sizeof(int), s);
        k_syrk_f64<<<nt * (nt + 1) / 2, 256, 0, s>>>(d_states, n, washout, T, A, n);
        k_add_diag<<<(n + 255) / 256, 256, 0, s>>>(A, n, n, lambda);
        if (lu_factor_solve(s, A, n, piv, info, W, dout) != 0) {
            // singular system: d_w_out is not written, and the caller is told
            cudaStreamSynchronize(s);
            return SP_EINTERNAL;
        }
    } else {
        chol_solve(s, A, n, W, dout);
    }
    const double bnorm = device_norm(s, B, tot, tmp);
    for (int it = 0;; ++it) {
        ridge_residual(s, d_states, n, washout, T, d_targets, W, dout, lambda, E, part, parts, R);
        const double rel = device_norm(s, R, tot, tmp) / (bnorm > 0 ? bnorm : 1.0);
        if (rel <= tol || it >= (lu ? 0 : maxit))
            break;
        chol_solve(s, A, n, R, dout);
        k_axpy<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(W, R, tot);
    }
    k_transpose_w<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(W, n, dout, d_w_out);
    if (cudaStreamSynchronize(s) != cudaSuccess || cudaGetLastError() != cudaSuccess)
        return SP_EINTERNAL;
    return SP_OK;
}
