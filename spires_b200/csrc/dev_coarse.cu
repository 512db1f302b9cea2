// dev_coarse.cu -- the merge loop of spires_coarse_grain on the device.
//
// Reference: coarse_grain_reservoir, src/reservoir.c:782-967. Pairs (i, j),
// j > i, are visited in row-major order; a pair is merged when W[i][j] or
// W[j][i] exceeds the threshold: V[i] = (V[i] + V[j]) / 2, V[j] = 0, row and
// column i become the pairwise combination of rows i and j (their sum where
// one of them is zero, else their mean), W_in row i likewise, W_out column j is
// added to column i, and row and column j are cleared. Full passes repeat
// until one merges nothing. Every merge changes the pairs tested after it, so
// the visiting order is kept exactly; what runs in parallel is the search for
// the next pair to merge along a row and the O(n) updates of each merge.
//
// One CTA of 1024 threads runs the whole loop in a single launch. The dense W
// and its transpose WT (WT[x][y] = W[y][x]) are kept in device memory, so the
// test of pair (i, j) reads row i of both with coalesced loads: the first j
// of a row that passes is found 4096 candidates at a time (4 per thread,
// loaded together, then a block-wide minimum). Arithmetic is IEEE double with
// the reference's operation order (_rn intrinsics, no contraction), so the
// merged matrices are bit-identical to the host loop's.
//
// The loop ends: every pass that merges kills a live neuron (thresholds are
// required to be >= 0, so a cleared row never passes again), hence at most
// n + 1 passes.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstring>
#include "sp_alloc.h"
#include "sp_kernels.cuh"
#include "sp_model.h"
#include "sp_dev.h"

namespace {

constexpr int kThreads = 1024;
constexpr int kPer = 4;  // candidates per thread per search round

__device__ __forceinline__ double combine(double a, double b)
{
    // (a * b == 0) ? a + b : (a + b) / 2, src/reservoir.c:870-873
    return sp::mul(a, b) == 0.0 ? sp::add(a, b) : sp::dvd(sp::add(a, b), 2.0);
}

__global__ void __launch_bounds__(kThreads, 1)
    k_coarse_merge(int n, int nin, int nout, double thr, double *W, double *WT, double *Win,
                   double *Wout, double *V, int *alive, long long *stats)
{
    __shared__ int s_first;
    __shared__ int s_merged;
    const int tid = threadIdx.x;
    const size_t N = (size_t)n;
    long long merges = 0, passes = 0;
    for (;;) {
        if (tid == 0)
            s_merged = 0;
        __syncthreads();
        ++passes;
        for (int i = 0; i < n; ++i) {
            const double *wi = W + (size_t)i * N;
            const double *wti = WT + (size_t)i * N;
            int j0 = i + 1;
            while (j0 < n) {
                // first j >= j0 with W[i][j] > thr || W[j][i] > thr
                int found = n;
                for (int base = j0; base < n && found == n; base += kThreads * kPer) {
                    if (tid == 0)
                        s_first = n;
                    __syncthreads();
                    double a[kPer], b[kPer];
#pragma unroll
                    for (int q = 0; q < kPer; ++q) {
                        const int j = base + q * kThreads + tid;
                        a[q] = j < n ? wi[j] : 0.0;
                        b[q] = j < n ? wti[j] : 0.0;
                    }
#pragma unroll
                    for (int q = 0; q < kPer; ++q) {
                        const int j = base + q * kThreads + tid;
                        if (j < n && (a[q] > thr || b[q] > thr)) {
                            atomicMin(&s_first, j);
                            break;
                        }
                    }
                    __syncthreads();
                    found = s_first;
                    __syncthreads();
                }
                if (found >= n)
                    break;
                const int j = found;
                ++merges;
                if (tid == 0) {
                    s_merged = 1;
                    V[i] = sp::dvd(sp::add(V[i], V[j]), 2.0);
                    V[j] = 0.0;
                    alive[j] = 0;
                }
                double *wj = W + (size_t)j * N;
                for (int k = tid; k < n; k += kThreads) {
                    if (k == i || k == j)
                        continue;
                    const double nw = combine(W[(size_t)i * N + k], wj[k]);
                    W[(size_t)i * N + k] = nw;
                    W[(size_t)k * N + i] = nw;
                    WT[(size_t)k * N + i] = nw;
                    WT[(size_t)i * N + k] = nw;
                }
                for (int k = tid; k < nin; k += kThreads) {
                    Win[(size_t)i * nin + k] = combine(Win[(size_t)i * nin + k],
                                                       Win[(size_t)j * nin + k]);
                    Win[(size_t)j * nin + k] = 0.0;
                }
                for (int o = tid; o < nout; o += kThreads) {
                    Wout[(size_t)o * N + i] = sp::add(Wout[(size_t)o * N + i], Wout[(size_t)o * N + j]);
                    Wout[(size_t)o * N + j] = 0.0;
                }
                __syncthreads();
                for (int k = tid; k < n; k += kThreads) {
                    W[(size_t)j * N + k] = 0.0;
                    W[(size_t)k * N + j] = 0.0;
                    WT[(size_t)k * N + j] = 0.0;
                    WT[(size_t)j * N + k] = 0.0;
                }
                __syncthreads();
                j0 = j + 1;
            }
        }
        __syncthreads();
        const int again = s_merged;
        __syncthreads();
        if (!again)
            break;
    }
    if (tid == 0) {
        stats[0] = merges;
        stats[1] = passes;
    }
}

__global__ void k_transpose(const double *__restrict__ A, int n, double *__restrict__ B)
{
    __shared__ double t[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int y = by + r, x = bx + threadIdx.x;
        t[r][threadIdx.x] = (y < n && x < n) ? A[(size_t)y * n + x] : 0.0;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int y = bx + r, x = by + threadIdx.x;
        if (y < n && x < n)
            B[(size_t)y * n + x] = t[threadIdx.x][r];
    }
}

}  // namespace

// In place on host arrays: W [n][n], Win [n][nin], Wout [nout][n], V [n],
// alive [n] (all 1 on entry). Returns an SP_* status.
extern "C" int sp_coarse_merge_device(size_t n, size_t nin, size_t nout, double thr, double *W,
                                      double *Win, double *Wout, double *V, int *alive)
{
    if (n == 0)
        return SP_OK;
    if (n > 65535 || !(thr >= 0.0))
        return SP_EINVAL;
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
        return SP_EINTERNAL;
    const size_t nn = n * n;
    double *dW = nullptr, *dWT = nullptr, *dWin = nullptr, *dWout = nullptr, *dV = nullptr;
    int *dA = nullptr;
    long long *dS = nullptr;
    int rc = SP_OK;
    if (sp_cuda_malloc(&dW, nn * 8) != cudaSuccess || sp_cuda_malloc(&dWT, nn * 8) != cudaSuccess ||
        sp_cuda_malloc(&dWin, (n * nin ? n * nin : 1) * 8) != cudaSuccess ||
        sp_cuda_malloc(&dWout, (n * nout ? n * nout : 1) * 8) != cudaSuccess ||
        sp_cuda_malloc(&dV, n * 8) != cudaSuccess || sp_cuda_malloc(&dA, n * 4) != cudaSuccess ||
        sp_cuda_malloc(&dS, 2 * 8) != cudaSuccess) {
        cudaGetLastError();
        rc = SP_EALLOC;
    }
#define CK(x)                             \
    do {                                  \
        if (!rc && (x) != cudaSuccess)    \
            rc = SP_EINTERNAL;            \
    } while (0)
    CK(cudaMemcpyAsync(dW, W, nn * 8, cudaMemcpyHostToDevice, s));
    if (nin)
        CK(cudaMemcpyAsync(dWin, Win, n * nin * 8, cudaMemcpyHostToDevice, s));
    if (nout)
        CK(cudaMemcpyAsync(dWout, Wout, n * nout * 8, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(dV, V, n * 8, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(dA, alive, n * 4, cudaMemcpyHostToDevice, s));
    if (!rc) {
        const dim3 g((unsigned)((n + 31) / 32), (unsigned)((n + 31) / 32)), b(32, 8);
        k_transpose<<<g, b, 0, s>>>(dW, (int)n, dWT);
        k_coarse_merge<<<1, kThreads, 0, s>>>((int)n, (int)nin, (int)nout, thr, dW, dWT, dWin,
                                              dWout, dV, dA, dS);
        CK(cudaGetLastError());
    }
    CK(cudaMemcpyAsync(W, dW, nn * 8, cudaMemcpyDeviceToHost, s));
    if (nin)
        CK(cudaMemcpyAsync(Win, dWin, n * nin * 8, cudaMemcpyDeviceToHost, s));
    if (nout)
        CK(cudaMemcpyAsync(Wout, dWout, n * nout * 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(V, dV, n * 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(alive, dA, n * 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
#undef CK
    cudaStreamSynchronize(s);
    void *bufs[] = {dW, dWT, dWin, dWout, dV, dA, dS};
    for (void *p : bufs)
        if (p)
            sp_cuda_free(p);
    cudaStreamDestroy(s);
    return rc;
}
