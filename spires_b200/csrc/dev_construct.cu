// dev_construct.cu -- construction work moved to the device.
//
// Spectral radius of the recurrent CSR matrix by the reference's max-abs
// normalised power iteration (src/sparse.c:93-127: x0 = 1, y = W x,
// lambda = max_i |y_i|, x = y / lambda, stop when |lambda - lambda_old| < 1e-6
// or after 1000 iterations). Every quantity is computed with the same
// operations in the same order as the host loop: each row is summed by one
// thread in ascending edge order from +0 with separate IEEE multiplies and
// adds, the maximum is exact in any order, and the division is IEEE. So the
// result, and the weights rescaled by it, are bit-identical to the host's,
// at a small fraction of its time for reservoirs with millions of edges.
//
// One cooperative launch runs all iterations with two bounded grid barriers
// per iteration (after the matrix-vector product and after the update of x).
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include "sp_alloc.h"
#include "sp_dev.h"
#include "sp_kernels.cuh"
#include "sp_dev_internal.h"

using namespace sp;

namespace {

struct PIArgs {
    long long n;
    const long long *row_ptr;
    const int *col;
    const double *w;
    double *x, *y;
    unsigned long long *lam;  // [2] bit patterns of the running maximum
    unsigned *bar;
    int *err;
    double *out;              // [0] lambda, [1] iterations run
    int max_iter;
    double tol;
};

__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long *p)
{
    return *(const volatile unsigned long long *)p;
}

__global__ void __launch_bounds__(256) k_power_iter(PIArgs a)
{
    __shared__ int s_flag;
    __shared__ double s_max[8];
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long g0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned nbar = 0;
    for (long long i = g0; i < a.n; i += stride)
        a.x[i] = 1.0;
    if (!grid_barrier(a.bar, ++nbar * gridDim.x, a.err, -1, &s_flag))
        return;
    double lam_old = 0.0, lam_new = 0.0;
    int it = 0;
    for (; it < a.max_iter; ++it) {
        const int slot = it & 1;
        double lm = 0.0;
        // one warp per row: the lanes load 32 edges' terms at once, and every
        // lane adds them in ascending edge order from +0 (the same sum as a
        // sequential walk of the row), so long rows do not serialise loads
        const int lane = threadIdx.x & 31;
        for (long long i = g0 >> 5; i < a.n; i += stride >> 5) {
            double s = 0.0;
            const long long k0 = __ldg(a.row_ptr + i), k1 = __ldg(a.row_ptr + i + 1);
            for (long long base = k0; base < k1; base += 32) {
                const long long k = base + lane;
                const double t = k < k1 ? mul(__ldg(a.w + k), __ldcg(a.x + __ldg(a.col + k))) : 0.0;
                const int cnt = k1 - base < 32 ? (int)(k1 - base) : 32;
                for (int j = 0; j < cnt; ++j)
                    s = add(s, __shfl_sync(kFull, t, j));
            }
            if (lane == 0)
                a.y[i] = s;
            const double v = fabs(s);
            if (v > lm)  // NaN never wins, as in the host comparison
                lm = v;
        }
        for (int off = 16; off > 0; off >>= 1) {
            const double o = __shfl_xor_sync(kFull, lm, off);
            if (o > lm)
                lm = o;
        }
        if ((threadIdx.x & 31) == 0)
            s_max[threadIdx.x >> 5] = lm;
        __syncthreads();
        if (threadIdx.x == 0) {
            double bm = 0.0;
            for (int k = 0; k < (int)(blockDim.x >> 5); ++k)
                if (s_max[k] > bm)
                    bm = s_max[k];
            // non-negative doubles order like their bit patterns
            if (bm > 0.0)
                atomicMax(a.lam + slot, (unsigned long long)__double_as_longlong(bm));
        }
        if (!grid_barrier(a.bar, ++nbar * gridDim.x, a.err, it, &s_flag))
            return;
        lam_new = __longlong_as_double((long long)ld_volatile_u64(a.lam + slot));
        for (long long i = g0; i < a.n; i += stride)
            a.x[i] = dvd(__ldcg(a.y + i), lam_new);
        if (blockIdx.x == 0 && threadIdx.x == 0)
            a.lam[slot ^ 1] = 0ull;  // every reader of that slot passed the last barrier
        if (fabs(sub(lam_new, lam_old)) < a.tol)
            break;
        lam_old = lam_new;
        if (!grid_barrier(a.bar, ++nbar * gridDim.x, a.err, it, &s_flag))
            return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.out[0] = lam_new;
        a.out[1] = (double)(it < a.max_iter ? it + 1 : a.max_iter);
    }
}

}  // namespace

// Device spectral radius of an n x n CSR matrix (host arrays). Returns SP_OK
// with *out set, or an error (no device, allocation failure, kernel error)
// after which the caller computes it on the host.
extern "C" int sp_dev_spectral_radius(size_t n, const int64_t *row_ptr, const int32_t *col,
                                      const double *w, double *out)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return SP_EINTERNAL;
    }
    const size_t nnz = (size_t)row_ptr[n];
    int dev = 0, sms = 0, coop = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_power_iter, 256, 0);
    if (!coop || per_sm < 1)
        return SP_EINTERNAL;
    per_sm = per_sm > 2 ? 2 : per_sm;
    // a warp per row: enough CTAs for the rows' edges, at most a full grid
    long long blocks = ((long long)n + 255) / 256;
    const long long by_edges = ((long long)row_ptr[n] + 16383) / 16384;
    if (blocks < by_edges)
        blocks = by_edges;
    if (blocks > (long long)per_sm * sms)
        blocks = (long long)per_sm * sms;
    if (blocks < 1)
        blocks = 1;

    cudaStream_t s = nullptr;
    char *buf = nullptr;
    int rc = SP_OK;
    const size_t o_rp = 0, o_col = o_rp + ((n + 1) * 8 + 255) / 256 * 256,
                 o_w = o_col + ((nnz ? nnz : 1) * 4 + 255) / 256 * 256,
                 o_x = o_w + ((nnz ? nnz : 1) * 8 + 255) / 256 * 256,
                 o_y = o_x + ((n ? n : 1) * 8 + 255) / 256 * 256,
                 o_small = o_y + ((n ? n : 1) * 8 + 255) / 256 * 256, total = o_small + 256;
    // stream-ordered allocation: no device-wide synchronisation, so several
    // host threads building reservoirs at once do not serialise here
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
        sp_cuda_malloc_async(&buf, total, s) != cudaSuccess) {
        cudaGetLastError();
        if (s)
            cudaStreamDestroy(s);
        return SP_EALLOC;
    }
    PIArgs a;
    a.n = (long long)n;
    a.row_ptr = (const long long *)(buf + o_rp);
    a.col = (const int *)(buf + o_col);
    a.w = (const double *)(buf + o_w);
    a.x = (double *)(buf + o_x);
    a.y = (double *)(buf + o_y);
    a.lam = (unsigned long long *)(buf + o_small);
    a.out = (double *)(buf + o_small + 16);
    a.bar = (unsigned *)(buf + o_small + 32);
    a.err = (int *)(buf + o_small + 48);
    a.max_iter = 1000;
    a.tol = 1e-6;
    double h_out[2] = {0.0, 0.0};
    int h_err[2] = {0, 0};
    void *args[] = {&a};
    bool ok = cudaMemcpyAsync(buf + o_rp, row_ptr, (n + 1) * 8, cudaMemcpyHostToDevice, s) ==
                  cudaSuccess &&
              cudaMemcpyAsync(buf + o_col, col, nnz * 4, cudaMemcpyHostToDevice, s) ==
                  cudaSuccess &&
              cudaMemcpyAsync(buf + o_w, w, nnz * 8, cudaMemcpyHostToDevice, s) == cudaSuccess &&
              cudaMemsetAsync(buf + o_small, 0, 256, s) == cudaSuccess &&
              cudaLaunchCooperativeKernel((const void *)k_power_iter, dim3((unsigned)blocks),
                                          dim3(256), args, 0, s) == cudaSuccess &&
              cudaMemcpyAsync(h_out, a.out, sizeof(h_out), cudaMemcpyDeviceToHost, s) ==
                  cudaSuccess &&
              cudaMemcpyAsync(h_err, a.err, sizeof(h_err), cudaMemcpyDeviceToHost, s) ==
                  cudaSuccess &&
              cudaStreamSynchronize(s) == cudaSuccess;
    if (!ok) {
        sp_dev_note_error("spectral radius", (int)cudaGetLastError());
        rc = SP_EINTERNAL;
    } else if (h_err[0] != 0) {
        rc = SP_EINTERNAL;
    } else {
        *out = h_out[0];
    }
    sp_cuda_free_async(buf, s);
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    return rc;
}

// Device selection for host worker threads (a new thread starts on device 0).
extern "C" int sp_dev_current_device(void)
{
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    return d;
}

extern "C" void sp_dev_use_device(int d)
{
    if (d >= 0 && cudaSetDevice(d) != cudaSuccess)
        cudaGetLastError();
}
