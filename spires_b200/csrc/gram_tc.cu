// gram_tc.cu -- the ridge Gram Phi^T Phi on the tensor cores with split
// operands.
//
// The states Phi (FP64) are split per element as x = hi + lo with hi the
// low-precision rounding of x and lo the rounding of the remainder x - hi:
//     BF16X3  hi, lo in BF16 (8-bit significands, 16 bits together)
//     TF32X3  hi, lo in TF32 (11-bit significands, 22 bits together)
// and the Gram is accumulated in FP32 by three tensor-core products
//     G = hi^T hi + hi^T lo + lo^T hi            (lo^T lo is below the sum's
// rounding and is dropped). The products are plain dense GEMMs over the time
// axis, issued to cuBLAS (BF16 / TF32 inputs, FP32 compute); the split, the
// FP64 widening with symmetrisation and everything after it (FP64 Cholesky,
// iterative refinement with residuals from the FP64 Phi) are this library's.
// The refinement recovers the FP64 solution whenever cond(Phi^T Phi + lambda I)
// times the Gram's relative error (about 1e-5 for BF16X3, 1e-6 for TF32X3)
// is well below one; the ridge report states the residual reached.
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cublas_v2.h>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include "sp_alloc.h"
#include "sp_gram.h"
#include "sp_model.h"
#include "sp_dev.h"
#include "sp_dev_internal.h"

namespace {

__device__ __forceinline__ float round_tf32(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// hi/lo split of rows [0, tw) of X (tw x n, row-major), written transposed
// (n x tw: each neuron's series contiguous, the reduction axis innermost, as
// the tensor-core GEMM reads its operands best). 32 x 32 tiles via shared
// memory; H is __nv_bfloat16 (BF16X3) or float holding TF32 values (TF32X3).
template <typename H>
__global__ void k_split_t(const double *__restrict__ X, int n, size_t tw, H *__restrict__ hi,
                          H *__restrict__ lo)
{
    __shared__ double tile[32][33];
    const size_t tb = (size_t)blockIdx.y * 32, ib = (size_t)blockIdx.x * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const size_t t = tb + r, i = ib + threadIdx.x;
        tile[r][threadIdx.x] = (t < tw && i < (size_t)n) ? X[t * n + i] : 0.0;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const size_t i = ib + r, t = tb + threadIdx.x;
        if (i >= (size_t)n || t >= tw)
            continue;
        const double x = tile[threadIdx.x][r];
        if constexpr (sizeof(H) == 2) {
            const __nv_bfloat16 h = __double2bfloat16(x);
            hi[i * tw + t] = h;
            lo[i * tw + t] = __double2bfloat16(x - (double)__bfloat162float(h));
        } else {
            const float h = round_tf32((float)x);
            hi[i * tw + t] = h;
            lo[i * tw + t] = round_tf32((float)(x - (double)h));
        }
    }
}

// C (FP64, ldc) from the column-major FP32 Gram: the lower triangle, mirrored.
__global__ void k_widen_sym(const float *__restrict__ G, int n, double *__restrict__ C, int ldc)
{
    const size_t total = (size_t)n * n;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
         k += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(k / n), j = (int)(k % n);
        const int a = i > j ? i : j, b = i > j ? j : i;  // (a, b) in the lower triangle
        C[(size_t)i * ldc + j] = (double)G[(size_t)b * n + a];
    }
}

[[maybe_unused]] unsigned grid_for(size_t cnt)
{
    size_t b = (cnt + 255) / 256;
    return (unsigned)(b > 16384 ? 16384 : (b ? b : 1));
}

// one cuBLAS handle per device, created on first use
std::mutex g_mu;
cublasHandle_t g_handle[64];

cublasHandle_t handle_for_current_device()
{
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= 64)
        return nullptr;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_handle[d] && cublasCreate(&g_handle[d]) != CUBLAS_STATUS_SUCCESS)
        g_handle[d] = nullptr;
    return g_handle[d];
}

}  // namespace

extern "C" int sp_gram_bf16x3_available(void) { return handle_for_current_device() != nullptr; }

extern "C" int sp_gram_split(cudaStream_t s, int mode, const double *X, int n, size_t t0,
                             size_t t1, double *C, int ldc)
{
    if ((mode != 1 && mode != 2) || t1 < t0 || t1 - t0 > (size_t)65535 * 32)
        return SP_EINVAL;
    cublasHandle_t h = handle_for_current_device();
    if (!h)
        return SP_EINTERNAL;
    std::lock_guard<std::mutex> lk(g_mu);  // the handle's stream is per call
    const size_t tw = t1 > t0 ? t1 - t0 : 0;
    const size_t cnt = tw * (size_t)n;
    const size_t esz = mode == 1 ? 2 : 4;
    void *hi = nullptr, *lo = nullptr;
    float *G = nullptr;
    int rc = SP_OK;
    if (sp_cuda_malloc_async(&hi, (cnt ? cnt : 1) * esz, s) != cudaSuccess ||
        sp_cuda_malloc_async(&lo, (cnt ? cnt : 1) * esz, s) != cudaSuccess ||
        sp_cuda_malloc_async(&G, (size_t)n * n * sizeof(float), s) != cudaSuccess) {
        cudaGetLastError();
        rc = SP_EALLOC;
    }
    if (!rc) {
        const double *Xs = X + t0 * (size_t)n;
        const dim3 g((n + 31) / 32, (unsigned)((tw + 31) / 32)), blk(32, 8);
        if (mode == 1)
            k_split_t<__nv_bfloat16><<<g, blk, 0, s>>>(Xs, n, tw, (__nv_bfloat16 *)hi,
                                                         (__nv_bfloat16 *)lo);
        else
            k_split_t<float><<<g, blk, 0, s>>>(Xs, n, tw, (float *)hi, (float *)lo);
        if (cudaGetLastError() != cudaSuccess)
            rc = SP_EINTERNAL;
    }
    if (!rc && cublasSetStream(h, s) != CUBLAS_STATUS_SUCCESS)
        rc = SP_EINTERNAL;
    if (!rc) {
        // column-major view: the split arrays are tw x n (ld tw); G = X^T X
        const cudaDataType_t dt = mode == 1 ? CUDA_R_16BF : CUDA_R_32F;
        const cublasComputeType_t ct =
            mode == 1 ? CUBLAS_COMPUTE_32F : CUBLAS_COMPUTE_32F_FAST_TF32;
        const float one = 1.0f, zero = 0.0f;
        const void *A[3] = {hi, hi, lo}, *B[3] = {hi, lo, hi};
        for (int q = 0; q < 3 && !rc; ++q) {
            const cublasStatus_t st = cublasGemmEx(
                h, CUBLAS_OP_T, CUBLAS_OP_N, n, n, (int)tw, &one, A[q], dt, (int)tw, B[q], dt,
                (int)tw, q == 0 ? &zero : &one, G, CUDA_R_32F, n, ct, CUBLAS_GEMM_DEFAULT);
            if (st != CUBLAS_STATUS_SUCCESS) {
                fprintf(stderr, "spires: cublasGemmEx failed (%d)\n", (int)st);
                rc = SP_EINTERNAL;
            }
        }
    }
    if (!rc) {
        k_widen_sym<<<grid_for((size_t)n * n), 256, 0, s>>>(G, n, C, ldc);
        if (cudaGetLastError() != cudaSuccess)
            rc = SP_EINTERNAL;
    }
    if (hi)
        sp_cuda_free_async(hi, s);
    if (lo)
        sp_cuda_free_async(lo, s);
    if (G)
        sp_cuda_free_async(G, s);
    return rc;
}

extern "C" int sp_gram_bf16x3(cudaStream_t s, const double *X, int n, size_t t0, size_t t1,
                              double *C, int ldc)
{
    return sp_gram_split(s, 1, X, n, t0, t1, C, ldc);
}
