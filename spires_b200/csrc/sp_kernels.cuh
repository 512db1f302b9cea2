// sp_kernels.cuh -- device helpers shared by the CUDA translation units.
//
// Parity arithmetic: the reference evaluates its dynamics in IEEE double with
// round-to-nearest and no fused multiply-add (x86-64 without FMA). Every
// operation on the parity path below goes through the explicit _rn
// intrinsics, which nvcc never contracts, so each product and each sum is
// rounded exactly once, in source order.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace sp {

constexpr unsigned kFull = 0xffffffffu;

// A kernel's dynamic shared-memory limit is one attribute per function for
// the whole process: reservoirs and batches built on other host threads share
// it, so a caller that set it to its own size could lower it under another
// caller's pending launch ("invalid argument"). Every caller therefore sets
// the same value, the device's opt-in maximum less the kernel's static shared
// memory; occupancy and launches still use each launch's own size.
inline cudaError_t set_max_dynamic_smem(const void *fn)
{
    int dev = 0, v = 0;
    cudaFuncAttributes fa;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e == cudaSuccess)
        e = cudaFuncGetAttributes(&fa, fn);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 v - (int)fa.sharedSizeBytes);
    return e;
}

__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }

__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_volatile_u32(const unsigned *p)
{
    return *(const volatile unsigned *)p;
}

__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long *p)
{
    return *(const volatile unsigned long long *)p;
}

__device__ __forceinline__ int ld_volatile_i32(const int *p)
{
    return *(const volatile int *)p;
}

// Error codes written to err[0] by device code; err[1] (and, where the step
// kernel records it, err[2]) hold the micro-step.
enum : int { kErrNone = 0, kErrBarrierTimeout = 1, kErrAborted = 2 };

// How long a CTA waits at a grid barrier before it gives up (the host then
// reports SPIRES_ERR_INTERNAL). Far above any legitimate wait.
constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;  // 2 s
constexpr unsigned long long kBarrierMaxPolls = 1ull << 31;

// Grid-wide barrier for a cooperative launch: every CTA adds one to *bar and
// waits until it reaches `target` (= (barrier index + 1) * gridDim.x). The
// wait is bounded; on timeout the CTA records the error and the whole grid
// returns. Returns false when the kernel must stop.
__device__ __forceinline__ bool grid_barrier(unsigned *bar, unsigned target, int *err,
                                             long long step, int *s_flag)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        __threadfence();
        atomicAdd(bar, 1u);
        if (ld_volatile_u32(bar) < target) {
            unsigned long long t0 = globaltimer_ns();
            unsigned long long polls = 0;
            while (ld_volatile_u32(bar) < target) {
                if (ld_volatile_i32(err) != kErrNone) {
                    ok = 0;
                    break;
                }
                if ((++polls & 255ull) == 0) {
                    if (globaltimer_ns() - t0 > kBarrierTimeoutNs || polls > kBarrierMaxPolls) {
                        if (atomicCAS(err, kErrNone, kErrBarrierTimeout) == kErrNone)
                            err[1] = (int)step;
                        ok = 0;
                        break;
                    }
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        *s_flag = ok;
    }
    __syncthreads();
    return *s_flag != 0;
}

// SplitMix64 (Steele, Lea, Flood 2014; the constants of Vigna's reference
// implementation), used for the FLIF_DIFFUSIVE refractory sampler.
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long *x)
{
    unsigned long long z = (*x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ double u01(unsigned long long *s)
{
    return (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0);
}

}  // namespace sp
