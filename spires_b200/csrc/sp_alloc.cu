// sp_alloc.cu -- counted device allocations and the allocation-failure test
// hook (sp_alloc.h).
#include <atomic>
#include "sp_alloc.h"

namespace {
std::atomic<long long> g_live{0};
// allocations still allowed before the injected failure; -1 = no failure
std::atomic<long long> g_fail_after{-1};

bool injected_failure()
{
    long long left = g_fail_after.load();
    while (left >= 0) {
        if (g_fail_after.compare_exchange_weak(left, left - 1))
            return left == 0;
    }
    return false;
}
}  // namespace

extern "C" cudaError_t sp_cuda_malloc_bytes(void **p, size_t bytes)
{
    if (injected_failure()) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaSuccess)
        ++g_live;
    return e;
}

extern "C" cudaError_t sp_cuda_malloc_async_bytes(void **p, size_t bytes, cudaStream_t s)
{
    if (injected_failure()) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    cudaError_t e = cudaMallocAsync(p, bytes, s);
    if (e == cudaSuccess)
        ++g_live;
    return e;
}

extern "C" cudaError_t sp_cuda_free(void *p)
{
    if (!p)
        return cudaSuccess;
    --g_live;
    return cudaFree(p);
}

extern "C" cudaError_t sp_cuda_free_async(void *p, cudaStream_t s)
{
    if (!p)
        return cudaSuccess;
    --g_live;
    return cudaFreeAsync(p, s);
}

extern "C" void sp_alloc_fail_after(long long count) { g_fail_after.store(count < 0 ? -1 : count); }

extern "C" long long sp_alloc_live(void) { return g_live.load(); }
