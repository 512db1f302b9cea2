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

// Stream-ordered allocations come from the device's default pool. Its release
// threshold is 0 by default, so every synchronisation hands freed blocks back
// to the driver and the next call maps them again (milliseconds for the
// hundreds of MB of Gram slices). Keep up to 8 GiB cached in the pool.
constexpr int kMaxDevices = 64;
std::atomic<int> g_pool_set[kMaxDevices];

void keep_pool(void)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return;
    }
    if (g_pool_set[dev].exchange(1))
        return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        unsigned long long thr = 8ull << 30;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    cudaGetLastError();
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
    keep_pool();
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
