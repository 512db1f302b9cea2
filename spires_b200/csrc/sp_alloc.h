// sp_alloc.h -- every device allocation of the library goes through these
// calls. They count the allocations that are live, and a test hook can make
// an allocation fail, so the failure paths of create, ridge and the other
// entry points can be exercised on the host side without touching the GPU.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>

extern "C" cudaError_t sp_cuda_malloc_bytes(void **p, size_t bytes);
extern "C" cudaError_t sp_cuda_malloc_async_bytes(void **p, size_t bytes, cudaStream_t s);
extern "C" cudaError_t sp_cuda_free(void *p);
extern "C" cudaError_t sp_cuda_free_async(void *p, cudaStream_t s);

template <class T>
static inline cudaError_t sp_cuda_malloc(T **p, size_t bytes)
{
    return sp_cuda_malloc_bytes((void **)p, bytes);
}

template <class T>
static inline cudaError_t sp_cuda_malloc_async(T **p, size_t bytes, cudaStream_t s)
{
    return sp_cuda_malloc_async_bytes((void **)p, bytes, s);
}
