// sp_gram.h -- mixed-precision Gram on the tensor cores (gram_tc.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstddef>

// 1 when the split tensor-core Gram can run on the current device.
extern "C" int sp_gram_bf16x3_available(void);

// C[n][n] (ldc) = sum_{t in [t0, t1)} X[t][:]^T X[t][:] with X (T x n, FP64,
// row-major) split as x = hi + lo (both BF16): hi*hi + hi*lo + lo*hi with FP32
// accumulation, written back as FP64. Returns an SP_* status.
extern "C" int sp_gram_bf16x3(cudaStream_t s, const double *X, int n, size_t t0, size_t t1,
                              double *C, int ldc);

// The same with mode 1 = BF16X3 or 2 = TF32X3 split operands.
extern "C" int sp_gram_split(cudaStream_t s, int mode, const double *X, int n, size_t t0,
                             size_t t1, double *C, int ldc);
