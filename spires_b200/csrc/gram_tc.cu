// gram_tc.cu -- the ridge Gram Phi^T Phi on the B200 tensor cores: this
// library's own sm_100a kernel (tcgen05.mma with TMEM accumulators, operands
// staged by TMA), replacing the FP64 SYRK where a mode asks for it.
//
// Reference: the Gram A = X^T X of train_output_ridge_regression
// (src/reservoir.c:615-623 -> mat_mat_mult, src/math_utils.c:154-162, one
// cblas_dgemm). The modes differ only in how an FP64 state is cut into
// tensor-core operands ("slices") and how the slice products are combined:
//
//   INT8 slices (mode 3; Ozaki, Ogita, Oishi, Rump, Numer. Algorithms 59, 2012,
//     error-free splitting with integer slices). Column i of the fitted states
//     is scaled by 2^-e_i (max_t |x_ti| < 2^e_i) and cut into k signed digits,
//     |d_s| <= 64: x = sum_s d_s 2^(-6-7(s-1)) + r, |r| <= 2^-7k. The Gram is
//     sum over digit pairs s + u <= k + 1 of d_s^T d_u 2^(-12-7(s+u-2)).
//     Every pair of one level s + u goes into one int32 TMEM accumulator (exact:
//     rows are taken in segments of at most 65472, so a level sum stays below
//     2^31); the epilogue combines the k level sums in FP64 from the smallest
//     level up and scales by 2^(e_i+e_j-12). k = 7 gives a Gram error at the
//     level of an FP64 dgemm (k = 8 below it), so the FP64 Cholesky and the
//     refinement that follow converge as they do on the FP64 Gram.
//   BF16X3 / TF32X3 (modes 1, 2): x = hi + lo, the products hi hi, hi lo,
//     lo hi accumulated in one FP32 TMEM accumulator; FP64 only afterwards
//     (Cholesky-preconditioned CG in the ridge solver).
//
// Layout. Slices are written K-major (time innermost) as [slice][n_pad][T_pad]
// by the split kernels; a CTA computes one 128 x 256 tile (rows I*128..,
// columns J*256..) of the lower triangle at a time, persistent over the tile
// list (N = 256: at N = 64 an MMA costs about as long as at N = 256, so the
// wider tile moves four times the work per instruction). Levels are taken one
// at a time, from the largest: per K chunk of 64 bytes a stage holds the A
// rows (2 TMA boxes of 64 rows x 64 B) and the B rows (4 boxes) of one digit
// pair, 64-byte swizzled, and two tcgen05.mma (K = 32 B each) add it into the
// level's 256-column TMEM accumulator; two accumulators alternate, so the
// epilogue drains one level while the next accumulates. The FP64 combination
// runs through the output (or a scratch for later row segments) in memory:
// the largest level written, each smaller one added, the last scaled by
// 2^(e_i+e_j-12) (tests/_ozaki_model.py restates the order in numpy).
// Warp 0 issues the TMA copies, warp 1 the MMAs (one thread), warps 2-5 drain
// TMEM (tcgen05.ld) and write FP64 rows. No cluster multicast is used.
//
// Every mbarrier wait is bounded (2 s): on timeout the kernel records an error,
// the roles stop, in-flight copies and MMAs are waited for (bounded), TMEM is
// freed and the host returns SP_EINTERNAL.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "sp_alloc.h"
#include "sp_kernels.cuh"
#include "sp_gram.h"
#include "sp_model.h"
#include "sp_dev.h"

namespace {

constexpr int kTileM = 128;                  // output tile rows
constexpr int kChunk = 64;                   // K bytes staged per chunk
constexpr int kBox = 64 * 64;                // one TMA box: 64 rows x 64 bytes
constexpr int kMaxSlices = 8, kMaxProd = 36;
constexpr int kSegChunks = 1023;             // int8: 1023 * 64 = 65472 rows per segment
constexpr int kThreads = 192;
constexpr unsigned long long kWaitNs = 2000000000ull;

// ------------------------------------------------------------ PTX helpers
__device__ __forceinline__ unsigned smem_u32(const void *p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ unsigned long long gtimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(unsigned long long *b, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned long long *b, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred P;\n mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n"
        " selp.u32 %0, 1, 0, P;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void mbar_arrive(unsigned long long *b)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *b, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y,
                                            unsigned long long *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_commit(unsigned long long *bar)
{
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_u32(bar))
        : "memory");
}

// Shared-memory matrix descriptor: K-major rows of 64 bytes, 64-byte swizzle,
// 8-row groups 512 bytes apart (stride byte offset), leading byte offset
// unused for a K extent inside one swizzle row; version 1 (sm_100).
__device__ __forceinline__ unsigned long long sdesc(unsigned saddr)
{
    unsigned long long d = 0;
    d |= (unsigned long long)((saddr & 0x3FFFFu) >> 4);
    d |= 1ull << 16;
    d |= (unsigned long long)(512 >> 4) << 32;
    d |= 1ull << 46;
    d |= 4ull << 61;
    return d;
}

template <int MODE>
__device__ __forceinline__ void mma(unsigned tmem_d, unsigned long long a, unsigned long long b,
                                    unsigned idesc, int accumulate)
{
    if constexpr (MODE == SP_GRAM_INT8) {
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
            "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
            : "memory");
    } else if constexpr (MODE == SP_GRAM_TF32X3) {
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
            "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
            : "memory");
    } else {
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
            "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
            : "memory");
    }
}

__device__ __forceinline__ void tmem_ld16(unsigned taddr, unsigned (&r)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
        "%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Bounded wait; false on timeout or when another role gave up.
__device__ __forceinline__ bool wait_bar(unsigned long long *b, unsigned parity, int *err,
                                         volatile int *s_abort, int where)
{
    if (mbar_try(b, parity))
        return true;
    const unsigned long long t0 = gtimer();
    unsigned polls = 0;
    while (!mbar_try(b, parity)) {
        if ((++polls & 63u) == 0) {
            if (*s_abort)
                return false;
            if (gtimer() - t0 > kWaitNs) {
                if (atomicCAS(err, 0, 1) == 0)
                    err[1] = where;
                *s_abort = 1;
                return false;
            }
        }
    }
    return true;
}

// ------------------------------------------------------- the Gram kernel
constexpr int kTileNL = 256;

struct GPL {
    int mode, nlev, nst, n, n_pad, tiles_i, ntiles, chunks, seg_chunks;
    unsigned idesc;
    signed char pa[kMaxProd], pb[kMaxProd];
    int lv_first[kMaxSlices + 1];  // products of level lv: [lv_first[lv], lv_first[lv + 1])
    const int *exps;
    double *C, *V;                 // output; per-segment sums of later row segments
    int ldc;
    int *err;
    alignas(64) CUtensorMap map;
};

// tile t -> (I, J): row block I (128 rows) has floor(I / 2) + 1 column blocks
// of 256 in the lower triangle
__device__ __forceinline__ void tile_ij_l(int t, int *I, int *J)
{
    int i = 0, base = 0;
    while (base + i / 2 + 1 <= t) {
        base += i / 2 + 1;
        ++i;
    }
    *I = i;
    *J = t - base;
}

template <int MODE>
__global__ void __launch_bounds__(kThreads, 1) k_gram_lv(const __grid_constant__ GPL p)
{
    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem =
        (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    constexpr int stage_bytes = 6 * kBox;  // A: 2 boxes (128 rows), B: 4 boxes (256 rows)
    unsigned long long *full = (unsigned long long *)(smem + (size_t)p.nst * stage_bytes);
    unsigned long long *empty = full + p.nst;
    unsigned long long *tfull = empty + p.nst;   // [2]
    unsigned long long *tempty = tfull + 2;      // [2]
    unsigned long long *mdone = tempty + 2;
    unsigned *tmem_slot = (unsigned *)(mdone + 1);
    __shared__ volatile int s_abort;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        s_abort = 0;
        for (int s = 0; s < p.nst; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], 4);
        }
        mbar_init(mdone, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(
                         smem_u32(tmem_slot))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = *tmem_slot;
    const int segs = (p.chunks + p.seg_chunks - 1) / p.seg_chunks;
    const int xstep = kChunk / (MODE == SP_GRAM_INT8 ? 1 : (MODE == SP_GRAM_BF16X3 ? 2 : 4));

    if (warp == 0) {
        // ---------------------------------------------------------- producer
        if (lane == 0) {
            long long q = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < p.ntiles && ok; t += gridDim.x) {
                int I, J;
                tile_ij_l(t, &I, &J);
                for (int sg = 0; sg < segs && ok; ++sg) {
                    const int c0 = sg * p.seg_chunks;
                    const int c1 = (c0 + p.seg_chunks < p.chunks) ? c0 + p.seg_chunks : p.chunks;
                    for (int lv = p.nlev - 1; lv >= 0 && ok; --lv) {
                        for (int k = p.lv_first[lv]; k < p.lv_first[lv + 1] && ok; ++k) {
                            const int rowA = p.pa[k] * p.n_pad + I * kTileM;
                            const int rowB = p.pb[k] * p.n_pad + J * kTileNL;
                            for (int c = c0; c < c1; ++c, ++q) {
                                const int st = (int)(q % p.nst);
                                const long long round = q / p.nst;
                                if (round > 0 &&
                                    !wait_bar(&empty[st], (unsigned)((round - 1) & 1), p.err,
                                              &s_abort, 1)) {
                                    ok = false;
                                    break;
                                }
                                unsigned char *A = smem + (size_t)st * stage_bytes;
                                mbar_expect_tx(&full[st], (unsigned)stage_bytes);
                                for (int b = 0; b < 2; ++b)
                                    tma_load_2d(A + b * kBox, &p.map, c * xstep, rowA + 64 * b,
                                                &full[st]);
                                for (int b = 0; b < 4; ++b)
                                    tma_load_2d(A + (2 + b) * kBox, &p.map, c * xstep,
                                                rowB + 64 * b, &full[st]);
                            }
                        }
                    }
                }
            }
            const unsigned long long t0 = gtimer();
            for (long long qq = (q > p.nst ? q - p.nst : 0); qq < q; ++qq) {
                const int st = (int)(qq % p.nst);
                while (!mbar_try(&full[st], (unsigned)((qq / p.nst) & 1)))
                    if (gtimer() - t0 > kWaitNs)
                        break;
            }
        }
    } else if (warp == 1) {
        // -------------------------------------------------------------- MMA
        if (lane == 0) {
            long long q = 0, pass = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < p.ntiles && ok; t += gridDim.x) {
                for (int sg = 0; sg < segs && ok; ++sg) {
                    const int c0 = sg * p.seg_chunks;
                    const int c1 = (c0 + p.seg_chunks < p.chunks) ? c0 + p.seg_chunks : p.chunks;
                    for (int lv = p.nlev - 1; lv >= 0 && ok; --lv, ++pass) {
                        const int buf = (int)(pass & 1);
                        if (pass >= 2 && !wait_bar(&tempty[buf], (unsigned)(((pass >> 1) - 1) & 1),
                                                   p.err, &s_abort, 2)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        const unsigned td = tmem + (unsigned)(buf * kTileNL);
                        for (int k = p.lv_first[lv]; k < p.lv_first[lv + 1] && ok; ++k) {
                            for (int c = c0; c < c1; ++c, ++q) {
                                const int st = (int)(q % p.nst);
                                if (!wait_bar(&full[st], (unsigned)((q / p.nst) & 1), p.err,
                                              &s_abort, 3)) {
                                    ok = false;
                                    break;
                                }
                                tc_fence_after();
                                const unsigned a0 = smem_u32(smem + (size_t)st * stage_bytes);
                                const unsigned b0 = a0 + 2 * kBox;
                                const bool first = (k == p.lv_first[lv]) && (c == c0);
#pragma unroll
                                for (int kk = 0; kk < 2; ++kk)
                                    mma<MODE>(td, sdesc(a0 + kk * 32), sdesc(b0 + kk * 32),
                                              p.idesc, !(first && kk == 0));
                                tc_commit(&empty[st]);
                            }
                        }
                        if (ok)
                            tc_commit(&tfull[buf]);
                    }
                }
            }
            tc_commit(mdone);
            const unsigned long long t0 = gtimer();
            while (!mbar_try(mdone, 0))
                if (gtimer() - t0 > kWaitNs)
                    break;
        }
        __syncwarp();
    } else {
        // --------------------------------------------------------- epilogue
        const int qd = warp & 3;
        const int r = qd * 32 + lane;
        long long pass = 0;
        bool ok = true;
        for (int t = blockIdx.x; t < p.ntiles && ok; t += gridDim.x) {
            int I, J;
            tile_ij_l(t, &I, &J);
            const int i = I * kTileM + r;
            const int ei = (MODE == SP_GRAM_INT8 && i < p.n_pad) ? __ldg(p.exps + i) : 0;
            for (int sg = 0; sg < segs && ok; ++sg) {
                double *vb = sg == 0 ? p.C : p.V;
                for (int lv = p.nlev - 1; lv >= 0 && ok; --lv, ++pass) {
                    const int buf = (int)(pass & 1);
                    int okw = 1;
                    if (lane == 0)
                        okw = wait_bar(&tfull[buf], (unsigned)((pass >> 1) & 1), p.err, &s_abort,
                                       4)
                                  ? 1
                                  : 0;
                    okw = __shfl_sync(0xffffffffu, okw, 0);
                    if (!okw) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const double sl = MODE == SP_GRAM_INT8 ? ldexp(1.0, -7 * lv) : 1.0;
                    const bool firstlv = lv == p.nlev - 1, lastlv = lv == 0;
                    for (int cc = 0; cc < kTileNL / 16; ++cc) {
                        unsigned a[16];
                        tmem_ld16(tmem + ((unsigned)(qd * 32) << 16) +
                                      (unsigned)(buf * kTileNL + cc * 16),
                                  a);
                        if (i >= p.n)
                            continue;
                        double *vrow = vb + (size_t)i * p.ldc;
                        double *crow = p.C + (size_t)i * p.ldc;
#pragma unroll
                        for (int c = 0; c < 16; ++c) {
                            const int j = J * kTileNL + cc * 16 + c;
                            if (j >= p.n)
                                continue;
                            double v;
                            if (MODE == SP_GRAM_INT8) {
                                const double x = __dmul_rn((double)(int)a[c], sl);
                                v = firstlv ? x : __dadd_rn(vrow[j], x);
                            } else {
                                v = (double)__uint_as_float(a[c]);
                            }
                            if (!lastlv) {
                                vrow[j] = v;
                            } else {
                                if (MODE == SP_GRAM_INT8)
                                    v = ldexp(v, ei + __ldg(p.exps + j) - 12);
                                crow[j] = sg == 0 ? v : __dadd_rn(crow[j], v);
                            }
                        }
                    }
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0)
                        mbar_arrive(&tempty[buf]);
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem)
                     : "memory");
    }
}

// ------------------------------------------------------ operand preparation

// e[i] = exponent with max_t |x_ti| < 2^e[i] (0 for a zero column); e starts
// very negative and is raised by atomicMax from row parts; bad[0] = 1 when
// any fitted state is not finite.
__global__ void k_col_exp(const double *__restrict__ X, int n, size_t t0, size_t tw, int parts,
                          int *__restrict__ e, int *__restrict__ bad)
{
    const int i = blockIdx.x * 32 + (threadIdx.x & 31);
    const int py = blockIdx.y * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int np = parts * (blockDim.x >> 5);
    if (i >= n)
        return;
    double m = 0.0;
    int nf = 0;
    for (size_t t = py; t < tw; t += np) {
        const double x = X[(t0 + t) * n + i];
        if (!isfinite(x))
            nf = 1;
        m = fmax(m, fabs(x));
    }
    if (nf)
        bad[0] = 1;
    if (m > 0.0) {
        int ex;
        frexp(m, &ex);
        atomicMax(e + i, ex);
    }
}

// exponents start as the memset pattern 0x80808080 (far below any frexp
// exponent); a column that stayed there is all zeros
__global__ void k_exp_fix(int *e, int n_pad)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n_pad && e[i] < -100000)
        e[i] = 0;
}

// Integer slices of rows [t0, t0 + tw) of X, written K-major:
// S[s][i][t] (n_pad x T_pad per slice; padding is zero). A block takes 128
// rows x 32 columns through shared memory; each thread then cuts 4
// consecutive rows of one column and writes 4 digits of a slice as one
// 32-bit word (a warp writes 128 contiguous bytes per slice).
__global__ void __launch_bounds__(256) k_slice_i8(const double *__restrict__ X, int n, size_t t0,
                                                  size_t tw, int n_pad, size_t T_pad,
                                                  const int *__restrict__ e, int k,
                                                  signed char *__restrict__ S)
{
    __shared__ double tile[128][33];
    const size_t tb = (size_t)blockIdx.y * 128;
    const int ib = blockIdx.x * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int rr = ty; rr < 128; rr += 8) {
        const size_t t = tb + rr;
        const int i = ib + tx;
        tile[rr][tx] = (t < tw && i < n) ? X[(t0 + t) * n + i] : 0.0;
    }
    __syncthreads();
    const size_t slice = (size_t)n_pad * T_pad;
    for (int r = 0; r < 4; ++r) {
        const int il = ty + 8 * r;
        const int i = ib + il;
        const int ex = e[i];
        unsigned w[kMaxSlices];
#pragma unroll
        for (int q = 0; q < kMaxSlices; ++q)
            w[q] = 0u;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            double v = __dmul_rn(ldexp(tile[4 * tx + j][il], -ex), 64.0);
#pragma unroll
            for (int q = 0; q < kMaxSlices; ++q) {
                if (q < k) {
                    const double d = rint(v);
                    w[q] |= ((unsigned)(int)d & 0xffu) << (8 * j);
                    v = __dmul_rn(__dsub_rn(v, d), 128.0);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < kMaxSlices; ++q)
            if (q < k)
                *(unsigned *)(S + q * slice + (size_t)i * T_pad + tb + 4 * tx) = w[q];
    }
}

__device__ __forceinline__ float round_tf32(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// hi/lo split (BF16 or TF32 in FP32 containers), written K-major as
// S[0] = hi, S[1] = lo, each n_pad x T_pad (padding zero).
template <typename H>
__global__ void k_split_hl(const double *__restrict__ X, int n, size_t t0, size_t tw, int n_pad,
                           size_t T_pad, H *__restrict__ S)
{
    __shared__ double tile[32][33];
    const size_t tb = (size_t)blockIdx.y * 32;
    const int ib = blockIdx.x * 32;
    for (int rr = threadIdx.y; rr < 32; rr += blockDim.y) {
        const size_t t = tb + rr;
        const int i = ib + threadIdx.x;
        tile[rr][threadIdx.x] = (t < tw && i < n) ? X[(t0 + t) * n + i] : 0.0;
    }
    __syncthreads();
    const size_t slice = (size_t)n_pad * T_pad;
    for (int rr = threadIdx.y; rr < 32; rr += blockDim.y) {
        const int i = ib + rr;
        const size_t t = tb + threadIdx.x;
        const double x = tile[threadIdx.x][rr];
        if constexpr (sizeof(H) == 2) {
            const __nv_bfloat16 h = __double2bfloat16(x);
            S[(size_t)i * T_pad + t] = h;
            S[slice + (size_t)i * T_pad + t] = __double2bfloat16(x - (double)__bfloat162float(h));
        } else {
            const float h = round_tf32((float)x);
            S[(size_t)i * T_pad + t] = h;
            S[slice + (size_t)i * T_pad + t] = round_tf32((float)(x - (double)h));
        }
    }
}

// upper triangle from the lower one
__global__ void k_mirror(double *C, int n, int ldc)
{
    const size_t total = (size_t)n * n;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(q / n), j = (int)(q % n);
        if (j > i)
            C[(size_t)i * ldc + j] = C[(size_t)j * ldc + i];
    }
}

typedef CUresult (*encode_tiled_fn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                    const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                    const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                    CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

encode_tiled_fn encoder()
{
    static encode_tiled_fn enc = nullptr;
    if (!enc) {
        void *fp = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fp, cudaEnableDefault, &q) ==
                cudaSuccess &&
            fp)
            enc = (encode_tiled_fn)fp;
    }
    return enc;
}

int device_ok()
{
    int dev = 0, major = 0, minor = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
        return 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
    return major == 10 && minor == 0;
}

template <int MODE>
int launch_gram_lv(cudaStream_t s, GPL &q, size_t smem)
{
    auto fn = k_gram_lv<MODE>;
    if (smem > 48 * 1024 && sp::set_max_dynamic_smem((const void *)fn) != cudaSuccess)
        return SP_EINTERNAL;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = q.ntiles < sms ? q.ntiles : sms;
    fn<<<grid, kThreads, smem, s>>>(q);
    return cudaGetLastError() == cudaSuccess ? SP_OK : SP_EINTERNAL;
}

}  // namespace

extern "C" int sp_gram_tc_available(void) { return device_ok(); }
extern "C" int sp_gram_bf16x3_available(void) { return device_ok(); }

extern "C" int sp_gram_tc(cudaStream_t s, int mode, int slices, const double *X, int n,
                          size_t t0, size_t t1, double *C, int ldc)
{
    if (mode != SP_GRAM_BF16X3 && mode != SP_GRAM_TF32X3 && mode != SP_GRAM_INT8)
        return SP_EINVAL;
    if (n <= 0 || t1 < t0 || ldc < n)
        return SP_EINVAL;
    if (mode == SP_GRAM_INT8 && (slices < 2 || slices > kMaxSlices))
        return SP_EINVAL;
    if (!device_ok() || !encoder())
        return SP_EINTERNAL;
    const size_t tw = t1 - t0;
    const int esz = mode == SP_GRAM_INT8 ? 1 : (mode == SP_GRAM_BF16X3 ? 2 : 4);
    // rows padded to a multiple of 128 elements (whole K chunks in every mode,
    // whole row tiles for the split kernels)
    const size_t T_pad = ((tw ? tw : 1) + 127) / 128 * 128;
    if (T_pad * esz / kChunk > (size_t)INT_MAX)
        return SP_EINVAL;
    const int n_pad = (n + kTileNL - 1) / kTileNL * kTileNL;
    const int ns = mode == SP_GRAM_INT8 ? slices : 2;
    const int chunks = (int)(T_pad * esz / kChunk);

    GPL q;
    memset(&q, 0, sizeof(q));
    q.mode = mode;
    q.n = n;
    q.n_pad = n_pad;
    q.tiles_i = n_pad / kTileM;
    for (int I = 0; I < q.tiles_i; ++I)
        q.ntiles += I / 2 + 1;
    q.chunks = chunks;
    // int8 level sums: at most `slices` products of |d| <= 64 digits per row
    q.seg_chunks = mode == SP_GRAM_INT8 ? kSegChunks : chunks;
    q.C = C;
    q.ldc = ldc;
    // products: INT8 digit pairs (a, b) with a + b <= k - 1, level a + b,
    // grouped by level; split modes hi.hi, hi.lo, lo.hi into one level
    int np = 0;
    if (mode == SP_GRAM_INT8) {
        for (int lv = 0; lv < slices; ++lv) {
            q.lv_first[lv] = np;
            for (int a = 0; a <= lv; ++a) {
                q.pa[np] = (signed char)a;
                q.pb[np] = (signed char)(lv - a);
                ++np;
            }
        }
        q.nlev = slices;
    } else {
        const int A[3] = {0, 0, 1}, B[3] = {0, 1, 0};
        for (int k = 0; k < 3; ++k) {
            q.pa[k] = (signed char)A[k];
            q.pb[k] = (signed char)B[k];
        }
        np = 3;
        q.lv_first[0] = 0;
        q.nlev = 1;
    }
    q.lv_first[q.nlev] = np;
    // instruction descriptor: D format (F32 = 1, S32 = 2), A/B formats
    // (S8 = 1 for kind::i8, BF16 = 1 for kind::f16, TF32 = 2 for kind::tf32),
    // K-major A and B, N >> 3, M >> 4
    const unsigned cfmt = mode == SP_GRAM_INT8 ? 2u : 1u;
    const unsigned abfmt = mode == SP_GRAM_TF32X3 ? 2u : 1u;
    q.idesc = (cfmt << 4) | (abfmt << 7) | (abfmt << 10) | ((unsigned)(kTileNL >> 3) << 17) |
              ((unsigned)(kTileM >> 4) << 24);
    const int segs = (q.chunks + q.seg_chunks - 1) / q.seg_chunks;

    // a stage: A 128 rows (2 boxes) and B 256 rows (4 boxes) of one K chunk
    const size_t stage_bytes = (size_t)6 * kBox;
    int dev = 0, smem_max = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t fixed = 1024 + 256;
    long long nst = ((long long)smem_max - (long long)fixed) / (long long)stage_bytes;
    if (nst > 8)
        nst = 8;
    if (nst < 2)
        return SP_EINVAL;
    q.nst = (int)nst;
    const size_t smem = fixed + (size_t)nst * stage_bytes;

    void *S = nullptr;
    int *ex = nullptr, *flags = nullptr;
    double *V = nullptr;
    int rc = SP_OK;
    if (segs > 1 &&
        sp_cuda_malloc_async(&V, (size_t)n * ldc * sizeof(double), s) != cudaSuccess) {
        cudaGetLastError();
        return SP_EALLOC;
    }
    const size_t sbytes = (size_t)ns * n_pad * T_pad * esz;
    if (sp_cuda_malloc_async(&S, sbytes, s) != cudaSuccess ||
        sp_cuda_malloc_async(&ex, (size_t)n_pad * sizeof(int), s) != cudaSuccess ||
        sp_cuda_malloc_async(&flags, 4 * sizeof(int), s) != cudaSuccess) {
        cudaGetLastError();
        rc = SP_EALLOC;
    }
    int hflags[4] = {0, 0, 0, 0};
    if (!rc && cudaMemsetAsync(flags, 0, 4 * sizeof(int), s) != cudaSuccess)
        rc = SP_EINTERNAL;
    if (!rc) {
        const dim3 g(n_pad / 32, (unsigned)(T_pad / 32)), blk(32, 8);
        if (mode == SP_GRAM_INT8) {
            if (cudaMemsetAsync(ex, 0x80, (size_t)n_pad * sizeof(int), s) != cudaSuccess)
                rc = SP_EINTERNAL;
            if (!rc) {
                const int parts = 64;
                k_col_exp<<<dim3((n + 31) / 32, parts), 256, 0, s>>>(X, n, t0, tw, parts, ex,
                                                                      flags + 2);
                k_exp_fix<<<(n_pad + 255) / 256, 256, 0, s>>>(ex, n_pad);
                k_slice_i8<<<dim3(n_pad / 32, (unsigned)(T_pad / 128)), 256, 0, s>>>(
                    X, n, t0, tw, n_pad, T_pad, ex, slices, (signed char *)S);
            }
        } else if (mode == SP_GRAM_BF16X3) {
            k_split_hl<__nv_bfloat16><<<g, blk, 0, s>>>(X, n, t0, tw, n_pad, T_pad,
                                                         (__nv_bfloat16 *)S);
        } else {
            k_split_hl<float><<<g, blk, 0, s>>>(X, n, t0, tw, n_pad, T_pad, (float *)S);
        }
        if (!rc && cudaGetLastError() != cudaSuccess)
            rc = SP_EINTERNAL;
    }
    if (!rc) {
        const CUtensorMapDataType dt = mode == SP_GRAM_INT8 ? CU_TENSOR_MAP_DATA_TYPE_UINT8
                                       : mode == SP_GRAM_BF16X3 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                                : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
        cuuint64_t dims[2] = {(cuuint64_t)T_pad, (cuuint64_t)ns * n_pad};
        cuuint64_t strides[1] = {(cuuint64_t)T_pad * esz};
        cuuint32_t box[2] = {(cuuint32_t)(kChunk / esz), 64};
        cuuint32_t estr[2] = {1, 1};
        if (encoder()(&q.map, dt, 2, S, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            rc = SP_EINTERNAL;
    }
    if (!rc) {
        q.exps = ex;
        q.err = flags;
        q.V = V;
        if (mode == SP_GRAM_INT8)
            rc = launch_gram_lv<SP_GRAM_INT8>(s, q, smem);
        else if (mode == SP_GRAM_BF16X3)
            rc = launch_gram_lv<SP_GRAM_BF16X3>(s, q, smem);
        else
            rc = launch_gram_lv<SP_GRAM_TF32X3>(s, q, smem);
    }
    if (!rc) {
        k_mirror<<<1024, 256, 0, s>>>(C, n, ldc);
        if (cudaGetLastError() != cudaSuccess)
            rc = SP_EINTERNAL;
    }
    // one wait for everything: a wait that ran out in the kernel, or (INT8) a
    // state that is not finite, in which case the caller takes the FP64 Gram
    if (!rc) {
        if (cudaMemcpyAsync(hflags, flags, 4 * sizeof(int), cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            rc = SP_EINTERNAL;
        else if (hflags[0]) {
            if (getenv("SPIRES_DEBUG"))
                fprintf(stderr, "spires: Gram kernel wait ran out (role %d)\n", hflags[1]);
            rc = SP_EINTERNAL;
        } else if (mode == SP_GRAM_INT8 && hflags[2]) {
            rc = SP_EINVAL;
        }
    }
    if (S)
        sp_cuda_free_async(S, s);
    if (ex)
        sp_cuda_free_async(ex, s);
    if (flags)
        sp_cuda_free_async(flags, s);
    if (V)
        sp_cuda_free_async(V, s);
    return rc;
}

extern "C" int sp_gram_split(cudaStream_t s, int mode, const double *X, int n, size_t t0,
                             size_t t1, double *C, int ldc)
{
    return sp_gram_tc(s, mode, mode == SP_GRAM_INT8 ? SP_GRAM_INT8_SLICES : 0, X, n, t0, t1, C,
                      ldc);
}

extern "C" int sp_gram_bf16x3(cudaStream_t s, const double *X, int n, size_t t0, size_t t1,
                              double *C, int ldc)
{
    return sp_gram_tc(s, SP_GRAM_BF16X3, 0, X, n, t0, t1, C, ldc);
}

// Public entry point (spires_ext_gram_device): C = X^T X over rows [t0, T) of
// device states X [T][n], on `stream`, waiting for it before returning.
extern "C" __attribute__((visibility("default"))) int
spires_ext_gram_device(const double *d_X, size_t T, size_t n, size_t t0, int mode, int slices,
                       double *d_C, void *stream)
{
    if (!d_X || !d_C || n == 0 || n > (size_t)INT_MAX || t0 > T)
        return SP_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    int rc;
    if (mode == SP_GRAM_FP64)
        rc = sp_gram_fp64(s, d_X, (int)n, t0, T, d_C, (int)n);
    else
        rc = sp_gram_tc(s, mode, slices > 0 ? slices : SP_GRAM_INT8_SLICES, d_X, (int)n, t0, T,
                        d_C, (int)n);
    if (rc == SP_OK && cudaStreamSynchronize(s) != cudaSuccess)
        rc = SP_EINTERNAL;
    return rc;
}
