// sp_gram.h -- the ridge Gram on the tensor cores (gram_tc.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstddef>

// Gram modes (the values of spires_ext_gram_mode)
enum { SP_GRAM_FP64 = 0, SP_GRAM_BF16X3 = 1, SP_GRAM_TF32X3 = 2, SP_GRAM_INT8 = 3 };
// integer slices of the INT8 mode unless the caller asks for another count
#define SP_GRAM_INT8_SLICES 7

// 1 when the tensor-core Gram can run on the current device (sm_100).
extern "C" int sp_gram_tc_available(void);
extern "C" int sp_gram_bf16x3_available(void);

// C[n][n] (ldc) = sum_{t in [t0, t1)} X[t][:]^T X[t][:] for X (T x n, FP64,
// row-major) on the tensor cores: mode SP_GRAM_INT8 with `slices` (2..8)
// integer slices, or the BF16X3 / TF32X3 split (slices ignored). The full
// matrix is written (lower triangle computed, mirrored). Returns an SP_*
// status; SP_EINVAL for a state that is not finite (INT8 mode).
extern "C" int sp_gram_tc(cudaStream_t s, int mode, int slices, const double *X, int n,
                          size_t t0, size_t t1, double *C, int ldc);

// The same with the default slice count.
extern "C" int sp_gram_split(cudaStream_t s, int mode, const double *X, int n, size_t t0,
                             size_t t1, double *C, int ldc);
extern "C" int sp_gram_bf16x3(cudaStream_t s, const double *X, int n, size_t t0, size_t t1,
                              double *C, int ldc);

// The FP64 Gram of the ridge solver (dev_readout.cu), same contract.
extern "C" int sp_gram_fp64(cudaStream_t s, const double *X, int n, size_t t0, size_t t1,
                            double *C, int ldc);
