// dev_batch.cu -- many reservoirs in one persistent launch.
//
// A batch holds `count` independent reservoirs of uneven size, ring length,
// series length and model (LIF_DISCRETE or FLIF_GL, SIMPLE synapses). Each is
// built on the host exactly as spires_reservoir_create builds it after
// srand(seed_i), so its dynamics are those of the unbatched path, bit for bit.
//
// Work table. The host plans a static schedule: the cooperative grid of P CTAs
// (256 threads each) is cut into groups of consecutive CTAs; each group runs a
// list of instances one after another, all its CTAs on one instance at a time
// with a group-local grid barrier (a counter per group). An instance needs at
// least ceil(nw / 8) CTAs (one neuron per thread); instances are placed
// heaviest first on the group that finishes them earliest (list scheduling on
// an estimated time that takes both the history stream and the per-step
// latency floor into account).
//
// The launch sequence of a run (input upload, state reset, barrier reset, the
// cooperative kernel, the raster gather and download) is captured once into a
// CUDA graph and replayed while the series lengths stay the same.
#include <cuda_runtime.h>
#include <algorithm>
#include <chrono>
#include <functional>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <vector>
#include "sp_alloc.h"
#include "sp_dev.h"
#include "sp_kernels.cuh"
#include "sp_dev_internal.h"
#include "sp_step_kernel.cuh"

using namespace sp;

namespace {

constexpr int kBatchThreads = 256;  // 8 warps per CTA

struct BInst {
    int n, nw, rs, din, L, ntype, micro;
    long long nnz;  // recurrent edges (schedule cost model)
    int dense;      // recurrent input from column blocks (see rowpass_columns)
    const uint2 *cmo;   // [n][nw] {row bits, weight offset} per (column, row word)
    const double *cw;   // [nnz] weights in column order
    long long T;  // macro steps of the current run
    double a, b, c, d, e, f, g, dt, gamma, v_init, tprev_init;
    double *V, *tprev, *ring;
    unsigned *spk;  // [2][nw]
    const long long *row_ptr;
    const int *col;
    const double *w, *W_in, *coef;
    const int *nid_of, *pos_of;
    // layout of W_out and of the readout sums: the single-reservoir path's
    // (equal to nid_of / pos_of except for column-block instances)
    const int *nid_ro, *pos_ro;
    const double *u;       // [T][din]
    double *phi;           // [T][rs] position order, or null
    unsigned *raster;      // [T][nw] position order
    unsigned *raster_nat;  // [T][nw] neuron order
    double *V_nat;         // [n] final state, neuron order
};

struct BParams {
    const BInst *inst;
    const int *cta_group, *group_start, *group_size, *job_off, *jobs;
    unsigned long long *bar;  // one arrival counter per group
    int *err;
    int lmax;                 // longest FLIF_GL ring of the batch (coefficients in smem)
    int max_nw;               // most spike words of an instance
    int list_cap;             // largest column-block instance (spike list in smem)
};

constexpr int kHistChunk = 32;  // ring values in flight per thread (cost model)

constexpr int kHistC = 8;  // ring values per cp.async group and thread
// groups in flight per thread (6 or 8 need more shared memory than two CTAs
// per SM allow, and one CTA per SM halved the sweep's throughput)
constexpr int kHistS = 4;

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(smem)), "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// FLIF_GL history of column `ci` for lags 2..lim in ascending order, with the
// ring values copied asynchronously into this thread's own shared-memory
// slots (s_h[(stage * kHistC + j) * kBatchThreads + tid]) kHistS groups ahead,
// so kHistS * kHistC loads are in flight while the ordered add chain runs.
// Only the issuing thread reads its slots, so no block barrier is needed.
__device__ __forceinline__ double batch_history_async(double hist, const double *s_coef,
                                                      const double *ci, int rs, int L, int head,
                                                      int lim, double *s_h, int tid)
{
    if (lim < 2)
        return hist;
    int r = head - 2;  // ring row of the next lag to issue
    if (r < 0)
        r += L;
    const double *gp = ci + (size_t)r * rs;   // its element of this column
    const double *gtop = ci + (size_t)(L - 1) * rs;
    int kiss = 2;  // next lag to issue
    auto issue = [&](int stg) {
        double *dst = s_h + (size_t)stg * kHistC * kBatchThreads + tid;
        if (kiss + kHistC - 1 <= lim && r >= kHistC - 1) {
            // a whole group before the ring's wrap: fixed offsets, no tests
#pragma unroll
            for (int j = 0; j < kHistC; ++j) {
                cp_async8(dst + (size_t)j * kBatchThreads, gp);
                gp -= rs;
            }
            r -= kHistC;
            if (r < 0) {
                r += L;
                gp = gtop;
            }
        } else {
#pragma unroll
            for (int j = 0; j < kHistC; ++j) {
                if (kiss + j <= lim) {
                    cp_async8(dst + (size_t)j * kBatchThreads, gp);
                    if (r == 0) {
                        r = L - 1;
                        gp = gtop;
                    } else {
                        --r;
                        gp -= rs;
                    }
                }
            }
        }
        kiss += kHistC;
        cp_async_commit();
    };
#pragma unroll
    for (int q = 0; q < kHistS - 1; ++q)
        issue(q);
    int stg = 0;
    for (int k = 2; k <= lim; k += kHistC) {
        issue((stg + kHistS - 1) % kHistS);  // possibly an empty group
        cp_async_wait<kHistS - 1>();          // the group of lags k.. has landed
        const double *src = s_h + (size_t)stg * kHistC * kBatchThreads + tid;
        if (k + kHistC - 1 <= lim) {
#pragma unroll
            for (int j = 0; j < kHistC; ++j)
                hist = add(hist, mul(s_coef[k + j], src[(size_t)j * kBatchThreads]));
        } else {
#pragma unroll
            for (int j = 0; j < kHistC; ++j)
                if (k + j <= lim)
                    hist = add(hist, mul(s_coef[k + j], src[(size_t)j * kBatchThreads]));
        }
        stg = (stg + 1 == kHistS) ? 0 : stg + 1;
    }
    cp_async_wait<0>();
    return hist;
}

// SIMPLE-synapse row pass of one warp (rows [row0, row0 + 32), lane r owns
// row row0 + r) for long rows: the warp's contiguous edge range is scanned in
// blocks of 32 * U edges whose column indices and weights are loaded one block
// ahead, so U loads per lane are in flight instead of one. Within a block the
// sub-chunks are taken in ascending edge order and each spiking edge's weight
// is added by the owner lane of its row: exactly the non-zero terms of
// csr_row_dot (src/sparse.c:68-76) in order, as in the one-chunk row pass.
template <int U>
__device__ __forceinline__ double rowpass_simple_warp_deep(const long long *__restrict__ row_ptr,
                                                           const int *__restrict__ col,
                                                           const double *__restrict__ w,
                                                           const unsigned *s_spk, int row0,
                                                           int lane)
{
    const long long e0 = __ldg(row_ptr + row0);
    const long long e1 = __ldg(row_ptr + row0 + 32);
    const long long my_end = __ldg(row_ptr + row0 + lane + 1);
    double acc = 0.0;
    int cn[U];
    double wn[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const long long k = e0 + 32 * u + lane;
        cn[u] = k < e1 ? __ldg(col + k) : -1;
        wn[u] = k < e1 ? __ldg(w + k) : 0.0;
    }
    for (long long base = e0; base < e1; base += 32 * U) {
        int c[U];
        double wv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            c[u] = cn[u];
            wv[u] = wn[u];
            const long long k = base + 32 * (U + u) + lane;
            cn[u] = k < e1 ? __ldg(col + k) : -1;
            wn[u] = k < e1 ? __ldg(w + k) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const bool sp = c[u] >= 0 && ((s_spk[c[u] >> 5] >> (c[u] & 31)) & 1u);
            unsigned m = __ballot_sync(kFull, sp);
            while (m) {
                const int bpos = __ffs(m) - 1;
                m &= m - 1;
                const long long eb = base + 32 * u + bpos;
                const double wb = __shfl_sync(kFull, wv[u], bpos);
                const unsigned owner = __ballot_sync(kFull, my_end > eb);
                if (lane == __ffs(owner) - 1)
                    acc = add(acc, wb);
            }
        }
    }
    return acc;
}

// SIMPLE-synapse recurrent input from column blocks, for dense matrices.
// Bits of row word q (rows 32q..32q+31) of column j say which of those rows
// have an edge from neuron j; the block's weights are stored contiguously in
// row order from its offset. The lane of row i walks the list of spiking
// neurons in ascending order and adds w_ij where the bit is set: exactly the
// non-zero terms of csr_row_dot (src/sparse.c:68-76) in ascending column
// order, reading 8 bytes per spiking column per 32 rows instead of 12 bytes per
// stored edge. Blocks are fetched C columns ahead.
__device__ __forceinline__ double rowpass_columns(const uint2 *__restrict__ cmo,
                                                  const double *__restrict__ cw,
                                                  const int *s_list, int cnt, int nw, int q,
                                                  int lane)
{
    constexpr int C = 8;
    const unsigned below = (1u << lane) - 1u;
    double acc = 0.0;
    uint2 cur[C], nxt[C];
#pragma unroll
    for (int u = 0; u < C; ++u)
        cur[u] = u < cnt ? __ldg(cmo + (size_t)s_list[u] * nw + q) : make_uint2(0u, 0u);
    for (int t = 0; t < cnt; t += C) {
#pragma unroll
        for (int u = 0; u < C; ++u)
            nxt[u] = t + C + u < cnt ? __ldg(cmo + (size_t)s_list[t + C + u] * nw + q)
                                     : make_uint2(0u, 0u);
        double wv[C];
#pragma unroll
        for (int u = 0; u < C; ++u)
            wv[u] = ((cur[u].x >> lane) & 1u) ? __ldg(cw + cur[u].y + __popc(cur[u].x & below))
                                              : 0.0;
#pragma unroll
        for (int u = 0; u < C; ++u)
            if ((cur[u].x >> lane) & 1u)
                acc = add(acc, wv[u]);
#pragma unroll
        for (int u = 0; u < C; ++u)
            cur[u] = nxt[u];
    }
    return acc;
}

// Ascending list of the spiking positions from the CTA's spike words: each
// thread takes a contiguous range of words, a block scan of their bit counts
// gives its write offset. Returns the count (all threads).
__device__ __forceinline__ int spike_list(const unsigned *s_spk, int nw, int *s_list,
                                          int *s_warp)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int per = (nw + kBatchThreads - 1) / kBatchThreads;
    const int w0 = tid * per < nw ? tid * per : nw;
    const int w1 = w0 + per < nw ? w0 + per : nw;
    int c = 0;
    for (int wi = w0; wi < w1; ++wi)
        c += __popc(s_spk[wi]);
    int x = c;  // inclusive warp scan
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(kFull, x, off);
        if (lane >= off)
            x += y;
    }
    if (lane == 31)
        s_warp[warp] = x;
    __syncthreads();
    int base = x - c;
    for (int k = 0; k < warp; ++k)
        base += s_warp[k];
    int total = 0;
    for (int k = 0; k < kBatchThreads / 32; ++k)
        total += s_warp[k];
    for (int wi = w0; wi < w1; ++wi) {
        unsigned m = s_spk[wi];
        while (m) {
            s_list[base++] = wi * 32 + __ffs(m) - 1;
            m &= m - 1;
        }
    }
    __syncthreads();  // list complete; s_warp free again
    return total;
}

// One persistent cooperative launch over the whole batch. CTA c belongs to
// group cta_group[c] (or to none, then it returns at once); a group runs its
// job list in order, splitting each instance's warps evenly over its CTAs,
// and meets at its own counter between micro-steps. The per-neuron arithmetic
// is that of the single-reservoir kernel for LIF_DISCRETE / FLIF_GL with
// SIMPLE synapses (src/neurons/lif_discrete.c:22-34, src/neurons/flif_gl.c:50-100,
// src/synapses/simple.c:59-64, src/reservoir.c:113-165).
#ifdef SP_PHASE_STAMPS
// Debug builds only: per job slot of the work table, the global timer when the
// group's first CTA started and finished it, the group, its width and the
// instance (spires_dbg_batch_job_stamps copies them out).
constexpr int kJobStampCap = 4096;
__device__ unsigned long long g_sp_jobstamps[kJobStampCap * 5];
#endif

__global__ void __launch_bounds__(kBatchThreads, 2) k_batch(BParams p)
{
    extern __shared__ __align__(16) unsigned char s_dyn[];
    double *s_coef = (double *)s_dyn;                    // [lmax]
    unsigned *s_spk = (unsigned *)(s_coef + p.lmax);     // [max_nw]
    int *s_list = (int *)(s_spk + p.max_nw);             // [list_cap]
    // per-thread ring staging (FLIF_GL batches), 16-byte aligned
    double *s_h = (double *)(((uintptr_t)(s_list + p.list_cap) + 15) & ~(uintptr_t)15);
    __shared__ int s_flag, s_abort;
    __shared__ int s_warp[kBatchThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int grp = p.cta_group[blockIdx.x];
    if (grp < 0)
        return;  // CTA outside every group: takes part in no barrier
    const int rank = blockIdx.x - p.group_start[grp];
    const int gsize = p.group_size[grp];
    unsigned long long *bar = p.bar + grp;
    unsigned long long nbar = 0;
    if (tid == 0)
        s_abort = 0;

    auto arrive = [&]() {
        __syncthreads();
        if (tid == 0 && gsize > 1) {
            __threadfence();
            atomicAdd(bar, 1ull);
        }
    };
    auto wait = [&](long long step) -> bool {
        ++nbar;
        if (tid == 0) {
            int ok = !s_abort;
            if (ok && gsize > 1) {
                const unsigned long long target = nbar * (unsigned long long)gsize;
                unsigned long long t0 = globaltimer_ns(), polls = 0;
                while (ld_volatile_u64(bar) < target) {
                    if ((++polls & 255ull) == 0) {
                        if (ld_volatile_i32(p.err) != kErrNone) {
                            ok = 0;
                            break;
                        }
                        if (globaltimer_ns() - t0 > kBarrierTimeoutNs || polls > kBarrierMaxPolls) {
                            if (atomicCAS(p.err, kErrNone, kErrBarrierTimeout) == kErrNone)
                                p.err[1] = (int)step;
                            ok = 0;
                            break;
                        }
                    }
                    __nanosleep(32);
                }
                __threadfence();
            }
            s_flag = ok;
            if (!ok)
                s_abort = 1;
        }
        __syncthreads();
        return s_flag != 0;
    };

    for (int j = p.job_off[grp]; j < p.job_off[grp + 1]; ++j) {
        const BInst &I = p.inst[p.jobs[j]];
        const long long B = I.T * I.micro;
        if (B == 0)
            continue;  // no steps: no arrival either, the counts stay matched
#ifdef SP_PHASE_STAMPS
        if (rank == 0 && tid == 0 && j < kJobStampCap) {
            g_sp_jobstamps[j * 5 + 0] = globaltimer_ns();
            g_sp_jobstamps[j * 5 + 2] = (unsigned long long)grp;
            g_sp_jobstamps[j * 5 + 3] = (unsigned long long)gsize;
            g_sp_jobstamps[j * 5 + 4] = (unsigned long long)p.jobs[j];
        }
#endif
        const int nw = I.nw, rs = I.rs, L = I.L;
        const bool gl = I.ntype == SP_FLIF_GL;
        const int wb0 = (int)((long long)rank * nw / gsize);
        const int wb1 = (int)((long long)(rank + 1) * nw / gsize);
        const int gw = wb0 + warp;
        const bool wact = gw < wb1;
        const int i = gw * 32 + lane;
        const int nid = wact ? I.nid_of[i] : -1;
        const bool act = nid >= 0;
        __syncthreads();  // previous job's readers of s_coef are done
        if (gl)
            for (int k = tid; k < L; k += kBatchThreads)
                s_coef[k] = I.coef[k];
        double V = act ? I.V[i] : 0.0;
        double tprev = (act && gl) ? I.tprev[i] : 0.0;
        double vlast = (act && gl) ? I.ring[(size_t)(L - 1) * rs + i] : 0.0;
        int cur = 0;
        double ext = 0.0;
        arrive();  // also publishes s_coef to the CTA
        for (long long b = 0; b < B; ++b) {
            const long long s = b / I.micro;
            const int m = (int)(b % I.micro);
            if (m == 0) {
                // ext = 0 + gamma * sum_k W_in[i][k] u[k] (netlib dgemv order)
                ext = 0.0;
                if (act && I.din > 0 && I.gamma != 0.0) {
                    const double *ur = I.u + (size_t)s * I.din;
                    const double *wr = I.W_in + (size_t)i * I.din;
                    double t = 0.0;
                    for (int k = 0; k < I.din; ++k)
                        t = add(t, mul(ldg_na(wr + k), ldg_na(ur + k)));
                    ext = add(0.0, mul(I.gamma, t));
                }
            }
            bool integ = false;
            double hist = 0.0;
            int head = 0;
            if (gl) {
                head = (int)(b % L);
                integ = tprev > I.f;
                const int lim = (int)(b < L ? b : L - 1);
                if (act && integ) {
                    if (lim >= 1)
                        hist = add(hist, mul(s_coef[1], vlast));
                    hist = batch_history_async(hist, s_coef, I.ring + i, rs, L, head, lim,
                                               s_h, tid);
                }
            }
            if (!wait(b))
                return;
            for (int wi = tid; wi < nw; wi += kBatchThreads)
                s_spk[wi] = __ldcg(I.spk + (size_t)cur * nw + wi);
            __syncthreads();
            double rec = 0.0;
            if (I.dense) {
                const int cnt = spike_list(s_spk, nw, s_list, s_warp);
                if (wact)
                    rec = rowpass_columns(I.cmo, I.cw, s_list, cnt, nw, gw, lane);
            } else if (wact) {
                // warp-uniform choice: long edge ranges take the deep pipeline
                const long long span = __ldg(I.row_ptr + gw * 32 + 32) - __ldg(I.row_ptr + gw * 32);
                rec = span > 256 ? rowpass_simple_warp_deep<8>(I.row_ptr, I.col, I.w, s_spk,
                                                                gw * 32, lane)
                                 : rowpass_simple_warp(I.row_ptr, I.col, I.w, s_spk, gw * 32, 32,
                                                       lane);
            }
            bool fired = false;
            if (act) {
                const double in = add(ext, rec);
                if (!gl) {
                    V = add(add(mul(I.c, V), in), I.d);
                    if (V > I.b) {
                        V = I.a;
                        fired = true;
                    }
                } else {
                    if (integ) {
                        const double rhs = add(add(dvd(-sub(vlast, I.c), I.d), in), I.e);
                        V = sub(mul(I.g, rhs), hist);
                        if (V >= I.a) {
                            V = I.b;
                            fired = true;
                            tprev = 0.0;
                        }
                    } else {
                        V = I.b;
                    }
                    I.ring[(size_t)head * rs + i] = V;
                    vlast = V;
                    tprev = add(tprev, I.dt);
                }
            }
            const unsigned word = __ballot_sync(kFull, fired);
            if (wact && lane == 0)
                I.spk[(size_t)(cur ^ 1) * nw + gw] = word;
            if (m == I.micro - 1) {
                if (act && I.phi)
                    I.phi[(size_t)s * rs + i] = V;
                if (wact && lane == 0)
                    I.raster[(size_t)s * nw + gw] = word;
            }
            if (b + 1 < B)
                arrive();
            cur ^= 1;
        }
        if (act) {
            I.V[i] = V;
            if (gl)
                I.tprev[i] = tprev;
        }
#ifdef SP_PHASE_STAMPS
        if (rank == 0 && tid == 0 && j < kJobStampCap)
            g_sp_jobstamps[j * 5 + 1] = globaltimer_ns();
#endif
    }
}

// Reset every instance to its initial state: blockIdx.y = instance.
__global__ void k_batch_reset(const BInst *inst)
{
    const BInst &I = inst[blockIdx.y];
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t start = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (size_t q = start; q < (size_t)I.rs; q += stride) {
        const bool act = I.nid_of[q] >= 0;
        I.V[q] = act ? I.v_init : 0.0;
        if (I.ntype == SP_FLIF_GL)
            I.tprev[q] = I.tprev_init;
    }
    for (size_t q = start; q < 2 * (size_t)I.nw; q += stride)
        I.spk[q] = 0u;
    if (I.ntype == SP_FLIF_GL)
        for (size_t k = start; k < (size_t)I.L * I.rs; k += stride)
            I.ring[k] = I.v_init;
}

// out[t][q] = in[t][nid[q]] (0 at holes): states of a column-block instance
// (neuron order) in its readout layout.
__global__ void k_rows_to_layout(const double *__restrict__ in, int rs,
                                 const int *__restrict__ nid, size_t T, double *__restrict__ out)
{
    const size_t total = T * (size_t)rs;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
         k += (size_t)gridDim.x * blockDim.x) {
        const size_t t = k / rs;
        const int q = (int)(k % rs);
        const int i = nid[q];
        out[k] = i >= 0 ? in[t * rs + i] : 0.0;
    }
}

// Rasters and final states of every instance back in neuron order.
__global__ void k_batch_gather(const BInst *inst)
{
    const BInst &I = inst[blockIdx.y];
    const size_t words = (size_t)I.nw;
    const size_t total = (size_t)I.T * words * 32;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
         k += (size_t)gridDim.x * blockDim.x) {
        const size_t t = k / (words * 32);
        const int i = (int)(k % (words * 32));
        bool b = false;
        if (i < I.n) {
            const int q = I.pos_of[i];
            b = (I.raster[t * words + (q >> 5)] >> (q & 31)) & 1u;
        }
        const unsigned m = __ballot_sync(kFull, b);
        if ((threadIdx.x & 31) == 0)
            I.raster_nat[t * words + (i >> 5)] = m;
    }
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)I.n;
         i += (size_t)gridDim.x * blockDim.x)
        I.V_nat[i] = I.V[I.pos_of[i]];
}

}  // namespace


// ============================================================== host side ==

struct sp_batch {
    int device = 0, num_sms = 0, P = 0;
    int P_max = 0;      // CTAs of the grid at full occupancy (P <= P_max)
    int plan_mode = 0;  // schedule family (plan()): set by sp_batch_autotune
    size_t smem = 0;
    int lmax = 0;
    int max_nw = 1, list_cap = 0;
    cudaStream_t stream = nullptr;
    std::vector<sp_host_model> models;
    std::vector<BInst> inst;
    std::vector<double *> w_pos;  // per instance W_out [dout][rs], position space
    char *arena = nullptr;
    BInst *d_inst = nullptr;
    int *d_sched = nullptr;  // cta_group | group_start | group_size | job_off | jobs
    unsigned long long *d_bar = nullptr;
    int *d_err = nullptr;
    int ngroups = 0;
    std::vector<int> cta_group, group_start, group_size, job_off, jobs;
    // staging of one run shape (series lengths + whether states are kept)
    std::vector<long long> T;
    int want_phi = -1;
    size_t u_total = 0, ras_total = 0, v_total = 0, phi_total = 0;
    double *d_u = nullptr, *h_u = nullptr;
    unsigned *d_ras = nullptr, *d_ras_nat = nullptr, *h_ras = nullptr;
    double *d_vnat = nullptr, *h_vnat = nullptr;
    double *d_phi = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_ok = 0;  // 1 captured, -1 capture refused (direct launches), 0 not tried
    long long runs = 0;
};

#define BK(x)                                                                      \
    do {                                                                           \
        cudaError_t e_ = (x);                                                      \
        if (e_ != cudaSuccess) {                                                   \
            sp_dev_note_error(#x, e_);                                             \
            return (e_ == cudaErrorMemoryAllocation) ? SP_EALLOC : SP_EINTERNAL;   \
        }                                                                          \
    } while (0)

static void batch_free_run(sp_batch *b)
{
    if (b->graph)
        cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graph_ok = 0;
    void *dv[] = {b->d_u, b->d_ras, b->d_ras_nat, b->d_vnat, b->d_phi};
    for (void *p : dv)
        if (p)
            sp_cuda_free(p);
    void *hv[] = {b->h_u, b->h_ras, b->h_vnat};
    for (void *p : hv)
        if (p)
            cudaFreeHost(p);
    b->d_u = b->h_u = b->d_vnat = b->h_vnat = b->d_phi = nullptr;
    b->d_ras = b->d_ras_nat = b->h_ras = nullptr;
    b->T.clear();
    b->want_phi = -1;
}

extern "C" void sp_batch_destroy(sp_batch *b)
{
    if (!b)
        return;
    if (b->stream)
        cudaStreamSynchronize(b->stream);
    batch_free_run(b);
    void *d[] = {b->arena, b->d_inst, b->d_sched, b->d_bar, b->d_err};
    for (void *p : d)
        if (p)
            sp_cuda_free(p);
    for (auto &m : b->models)
        sp_model_free(&m);
    if (b->stream)
        cudaStreamDestroy(b->stream);
    delete b;
}

static int min_ctas(const BInst &I) { return (I.nw + kBatchThreads / 32 - 1) / (kBatchThreads / 32); }

// Estimated seconds for one instance on g CTAs: the larger of a per-step
// latency floor and the instance's share of the CTAs' streaming rate. The
// floor adds the barrier, the row pass (its warps scan 256 edges per memory
// round trip on long rows, 32 on short ones) and the FLIF_GL history (16 ring
// values per round trip); the bytes are the CSR scan (column + weight per
// edge), the history ring and the neuron state.
static double est_time(const BInst &I, long long T, int g)
{
    const double cta_bw = 20e9;   // bytes/s one CTA streams
    const double trip = 0.35e-6;  // one dependent memory round trip
    const double steps = (double)T * I.micro;
    const double span = (double)I.nnz / (I.nw > 0 ? I.nw : 1);  // edges per warp
    double rows = span > 256 ? std::ceil(span / 256.0) : std::ceil(span / 32.0);
    double bytes = 12.0 * (double)I.nnz + 24.0 * I.n;
    if (I.dense) {  // column blocks: about a tenth of the columns spike per step
        rows = std::ceil(0.1 * I.n / 8.0);
        bytes = 0.8 * I.n * (double)I.nw + 0.8 * (double)I.nnz + 24.0 * I.n;
    }
    double floor_s = 2e-6 + trip * rows;
    if (I.ntype == SP_FLIF_GL) {
        floor_s += trip * ((I.L + kHistChunk - 1) / kHistChunk);
        bytes += 8.0 * I.n * (double)I.L;
    }
    return steps * std::max(floor_s, bytes / (g * cta_bw));
}

// Static schedule: instances in the given order go to the existing group
// (wide enough) that finishes them first, or to a new group of their minimum
// width while CTAs are free. Returns false when an instance found no group.
static bool plan_order(sp_batch *b, const std::vector<int> &order, const std::vector<long long> &T)
{
    struct G {
        int start, size;
        double busy;
        std::vector<int> jobs;
    };
    std::vector<G> groups;
    int used = 0;
    for (int k : order) {
        const BInst &I = b->inst[k];
        const int gmin = min_ctas(I);
        int best = -1;
        double best_fin = 1e300;
        for (size_t gi = 0; gi < groups.size(); ++gi) {
            if (groups[gi].size < gmin)
                continue;
            const double fin = groups[gi].busy + est_time(I, T[k], groups[gi].size);
            if (fin < best_fin) {
                best_fin = fin;
                best = (int)gi;
            }
        }
        if (used + gmin <= b->P) {
            const double fin = est_time(I, T[k], gmin);
            if (best < 0 || fin < best_fin) {
                groups.push_back(G{used, gmin, 0.0, {}});
                used += gmin;
                best = (int)groups.size() - 1;
                best_fin = fin;
            }
        }
        if (best < 0)
            return false;
        groups[best].busy = best_fin;
        groups[best].jobs.push_back(k);
    }
    b->ngroups = (int)groups.size();
    b->cta_group.assign(b->P, -1);
    b->group_start.clear();
    b->group_size.clear();
    b->job_off.assign(1, 0);
    b->jobs.clear();
    for (size_t gi = 0; gi < groups.size(); ++gi) {
        for (int c = 0; c < groups[gi].size; ++c)
            b->cta_group[groups[gi].start + c] = (int)gi;
        b->group_start.push_back(groups[gi].start);
        b->group_size.push_back(groups[gi].size);
        for (int k : groups[gi].jobs)
            b->jobs.push_back(k);
        b->job_off.push_back((int)b->jobs.size());
    }
    return true;
}

// Heaviest first (longest-processing-time list scheduling); if a wide
// instance then finds every CTA taken by narrower groups, plan again widest
// first, which always succeeds because every instance fits the grid.
// Size-class schedule: every instance runs on a group whose width is its
// minimum CTA count rounded up to a power of two; each class gets one group,
// then the free CTAs go one group at a time to the class with the longest
// estimated time per group (balancing the classes' finish times), and each
// class's instances are dealt heaviest first to its least busy group.
// Many narrow groups keep every SM busy with instances that each run at their
// own per-step latency. Returns false when the classes do not fit the grid.
static bool plan_classes(sp_batch *b, const std::vector<long long> &T, int widen, bool pow2)
{
    const int P = b->P;
    const size_t cnt = b->inst.size();
    std::vector<int> width(cnt);
    std::vector<int> classes;
    for (size_t k = 0; k < cnt; ++k) {
        int w = 1;
        if (pow2) {
            while (w < min_ctas(b->inst[k]))
                w <<= 1;
        } else {
            w = min_ctas(b->inst[k]);
        }
        w *= widen;
        if (w > P)
            w = min_ctas(b->inst[k]);
        width[k] = w;
        if (std::find(classes.begin(), classes.end(), w) == classes.end())
            classes.push_back(w);
    }
    std::sort(classes.begin(), classes.end(), std::greater<int>());
    std::vector<double> work(classes.size(), 0.0);
    std::vector<int> members(classes.size(), 0);
    for (size_t k = 0; k < cnt; ++k) {
        const size_t c = std::find(classes.begin(), classes.end(), width[k]) - classes.begin();
        work[c] += est_time(b->inst[k], T[k], width[k]);
        members[c]++;
    }
    int need = 0;
    for (int w : classes)
        need += w;
    if (need > P)
        return false;
    double total = 0.0;
    for (double x : work)
        total += x;
    std::vector<int> ngroups(classes.size(), 1);
    int used = need;
    // hand out the remaining CTAs one group at a time to the class whose
    // time per group is longest
    for (;;) {
        int bestc = -1;
        double bestload = 0.0;
        for (size_t c = 0; c < classes.size(); ++c) {
            if (used + classes[c] > P || ngroups[c] >= members[c])
                continue;
            const double load = work[c] / ngroups[c];
            if (bestc < 0 || load > bestload) {
                bestload = load;
                bestc = (int)c;
            }
        }
        if (bestc < 0)
            break;
        ngroups[bestc]++;
        used += classes[bestc];
    }
    (void)total;
    struct G {
        int start, size;
        double busy;
        std::vector<int> jobs;
    };
    std::vector<G> groups;
    std::vector<int> first(classes.size());
    int start = 0;
    for (size_t c = 0; c < classes.size(); ++c) {
        first[c] = (int)groups.size();
        for (int q = 0; q < ngroups[c]; ++q) {
            groups.push_back(G{start, classes[c], 0.0, {}});
            start += classes[c];
        }
    }
    std::vector<int> order(cnt);
    std::iota(order.begin(), order.end(), 0);
    std::vector<double> est(cnt);
    for (size_t k = 0; k < cnt; ++k)
        est[k] = est_time(b->inst[k], T[k], width[k]);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return est[x] > est[y]; });
    for (int k : order) {
        const size_t c = std::find(classes.begin(), classes.end(), width[k]) - classes.begin();
        int best = first[c];
        for (int gi = first[c]; gi < first[c] + ngroups[c]; ++gi)
            if (groups[gi].busy < groups[best].busy)
                best = gi;
        groups[best].busy += est[k];
        groups[best].jobs.push_back(k);
    }
    b->ngroups = (int)groups.size();
    b->cta_group.assign(P, -1);
    b->group_start.clear();
    b->group_size.clear();
    b->job_off.assign(1, 0);
    b->jobs.clear();
    for (size_t gi = 0; gi < groups.size(); ++gi) {
        for (int q = 0; q < groups[gi].size; ++q)
            b->cta_group[groups[gi].start + q] = (int)gi;
        b->group_start.push_back(groups[gi].start);
        b->group_size.push_back(groups[gi].size);
        for (int k : groups[gi].jobs)
            b->jobs.push_back(k);
        b->job_off.push_back((int)b->jobs.size());
    }
    return true;
}

// Schedule families (b->plan_mode): 0 size classes of power-of-two widths,
// 1 size classes of the exact minimum widths, 2 size classes of twice the
// power-of-two widths (fewer, wider groups), 3 list scheduling heaviest first.
// Each falls back to list scheduling when its classes do not fit the grid.
static void plan(sp_batch *b, const std::vector<long long> &T)
{
    const int mode = b->plan_mode;
    if (mode == 0 && plan_classes(b, T, 1, true))
        return;
    if (mode == 1 && plan_classes(b, T, 1, false))
        return;
    if (mode == 2 && plan_classes(b, T, 2, true))
        return;
    const size_t cnt = b->inst.size();
    std::vector<int> order(cnt);
    std::iota(order.begin(), order.end(), 0);
    std::vector<double> solo(cnt);
    for (size_t k = 0; k < cnt; ++k)
        solo[k] = est_time(b->inst[k], T[k], min_ctas(b->inst[k]));
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return solo[x] > solo[y]; });
    if (plan_order(b, order, T))
        return;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        const int gx = min_ctas(b->inst[x]), gy = min_ctas(b->inst[y]);
        return gx != gy ? gx > gy : solo[x] > solo[y];
    });
    plan_order(b, order, T);
}

extern "C" int sp_batch_create(sp_host_model *models, size_t count, sp_batch **out)
{
    *out = nullptr;
    if (count == 0 || count > 65535)
        return SP_EINVAL;
    for (size_t k = 0; k < count; ++k) {
        const sp_host_model &m = models[k];
        if ((m.neuron_type != SP_LIF_DISCRETE && m.neuron_type != SP_FLIF_GL) ||
            m.syn_type != SP_SYN_SIMPLE || m.n == 0 || m.dout > 16)
            return SP_EINVAL;
    }
    sp_batch *b = new sp_batch();
    if (cudaGetDevice(&b->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete b;
        return SP_EINTERNAL;
    }
    cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, b->device);
    b->models.assign(models, models + count);
    memset(models, 0, count * sizeof(sp_host_model)); /* the batch owns the buffers now */

    size_t total = 0;
    auto take = [&](size_t bytes) {
        const size_t o = total;
        total += (bytes + 255) & ~(size_t)255;
        return o;
    };
    b->inst.resize(count);
    b->w_pos.resize(count);
    struct Off {
        size_t V, tp, ring, spk, rp, col, w, win, coef, nid, pos, wout, cmo, cw, nro, pro;
    };
    std::vector<Off> off(count);
    std::vector<std::vector<int>> pos(count), nid(count);
    size_t max_nw = 1;
    int list_cap = 0;
    for (size_t k = 0; k < count; ++k) {
        const sp_host_model &m = b->models[k];
        BInst &I = b->inst[k];
        memset(&I, 0, sizeof(I));
        I.n = (int)m.n;
        I.nw = (int)((m.n + 31) / 32);
        I.rs = I.nw * 32;
        I.din = (int)m.din;
        I.L = m.neuron_type == SP_FLIF_GL ? m.nc.L : 1;
        I.ntype = m.neuron_type;
        I.micro = m.micro_steps;
        I.nnz = (long long)m.nnz;
        // column blocks when at least one edge in 256 pairs is present (the
        // spike list of up to 16384 neurons fits shared memory)
        I.dense = m.nnz > 0 && (double)m.nnz * 256.0 >= (double)m.n * (double)m.n &&
                  m.n <= 16384 && m.nnz < 0xFFFFFFFFull;
        I.a = m.nc.a;
        I.b = m.nc.b;
        I.c = m.nc.c;
        I.d = m.nc.d;
        I.e = m.nc.e;
        I.f = m.nc.f;
        I.g = m.nc.g;
        I.dt = m.dt;
        I.gamma = m.input_strength;
        I.v_init = m.nc.v_init;
        I.tprev_init = m.nc.tprev_init;
        max_nw = std::max(max_nw, (size_t)I.nw);
        if (I.ntype == SP_FLIF_GL)
            b->lmax = std::max(b->lmax, I.L);
        const size_t rs = I.rs;
        Off &o = off[k];
        o.V = take(rs * 8);
        o.tp = take(rs * 8);
        o.ring = take(I.ntype == SP_FLIF_GL ? rs * (size_t)I.L * 8 : 8);
        o.spk = take(2 * (size_t)I.nw * 4);
        o.rp = take((rs + 1) * 8);
        o.col = take((I.dense || !m.nnz ? 1 : m.nnz) * 4);
        o.w = take((I.dense || !m.nnz ? 1 : m.nnz) * 8);
        o.cmo = take(I.dense ? (size_t)m.n * I.nw * 8 : 8);
        o.cw = take(I.dense ? m.nnz * 8 : 8);
        o.nro = take(I.dense ? rs * 4 : 8);
        o.pro = take(I.dense ? m.n * 4 : 8);
        if (I.dense)
            list_cap = std::max(list_cap, (int)m.n);
        o.win = take(rs * (m.din ? m.din : 1) * 8);
        o.coef = take((size_t)I.L * 8);
        o.nid = take(rs * 4);
        o.pos = take(m.n * 4);
        o.wout = take(rs * (m.dout ? m.dout : 1) * 8);
    }
    b->max_nw = (int)max_nw;
    b->list_cap = list_cap;
    b->smem = (size_t)b->lmax * 8 + max_nw * 4 + (size_t)list_cap * 4 + 16 +
              (b->lmax > 0 ? (size_t)kHistS * kHistC * kBatchThreads * 8 : 0);
    int rc = SP_OK;
    int per_sm = 0;
    if (b->smem > 200 * 1024)
        rc = SP_EINVAL;
    if (!rc && b->smem > 48 * 1024 && set_max_dynamic_smem((const void *)k_batch) != cudaSuccess)
        rc = SP_EINVAL;
    if (!rc) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch, kBatchThreads, b->smem);
        per_sm = std::min(per_sm, 2);
        if (per_sm < 1)
            rc = SP_EINVAL;
        b->P = per_sm * b->num_sms;
        b->P_max = b->P;
    }
    for (size_t k = 0; !rc && k < count; ++k)
        if (min_ctas(b->inst[k]) > b->P)
            rc = SP_EINVAL;  // wider than the whole grid
    if (!rc && sp_cuda_malloc(&b->arena, total) != cudaSuccess)
        rc = SP_EALLOC;
    if (rc) {
        cudaGetLastError();
        sp_batch_destroy(b);
        return rc;
    }
    // Layouts, position-order CSR and uploads of the instances on all host
    // threads (each worker thread selects the batch's device first).
    int failed = 0;
#pragma omp parallel for schedule(dynamic, 1)
    for (size_t k = 0; k < count; ++k) {
        if (failed)
            continue;
        cudaSetDevice(b->device);
        const sp_host_model &m = b->models[k];
        BInst &I = b->inst[k];
        const Off &o = off[k];
        char *A = b->arena;
        const size_t rs = I.rs;
        std::vector<int> pos_ro, nid_ro;  // readout layout of column-block instances
        if (I.dense) {
            // column blocks read spike lists in neuron order: identity layout;
            // W_out and the readout sums keep the single path's layout
            sp_make_layout(&m, I.nw, nullptr, pos_ro, nid_ro);
            pos[k].resize(m.n);
            nid[k].assign(rs, -1);
            for (size_t i = 0; i < m.n; ++i) {
                pos[k][i] = (int)i;
                nid[k][i] = (int)i;
            }
        } else {
            sp_make_layout(&m, I.nw, nullptr, pos[k], nid[k]);
        }
        // CSR in position order, as the single-reservoir path lays it out
        // (column-block instances keep only empty rows here)
        const size_t ecap = (I.dense || !m.nnz) ? 1 : m.nnz;
        std::vector<long long> rp(rs + 1, 0);
        std::vector<int> col(ecap);
        std::vector<double> w(ecap), win(rs * (m.din ? m.din : 1), 0.0),
            wout(rs * (m.dout ? m.dout : 1), 0.0);
        std::vector<uint2> cmo;
        std::vector<double> cw;
        if (I.dense) {
            // blocks (column j, row word q): row bits and the offset of the
            // block's weights, stored column by column in row order
            cmo.assign((size_t)m.n * I.nw, make_uint2(0u, 0u));
            cw.resize(m.nnz);
            std::vector<long long> cstart(m.n + 1, 0);
            for (size_t kk = 0; kk < m.nnz; ++kk)
                cstart[m.col[kk] + 1]++;
            for (size_t j = 0; j < m.n; ++j)
                cstart[j + 1] += cstart[j];
            std::vector<long long> fill(cstart.begin(), cstart.end() - 1);
            for (size_t i = 0; i < m.n; ++i)
                for (int64_t kk = m.row_ptr[i]; kk < m.row_ptr[i + 1]; ++kk) {
                    const int j = m.col[kk];
                    cw[fill[j]++] = m.w[kk];
                    cmo[(size_t)j * I.nw + i / 32].x |= 1u << (i % 32);
                }
            for (size_t j = 0; j < m.n; ++j) {
                long long run = cstart[j];
                for (int q = 0; q < I.nw; ++q) {
                    cmo[(size_t)j * I.nw + q].y = (unsigned)run;
                    run += __builtin_popcount(cmo[(size_t)j * I.nw + q].x);
                }
            }
        }
        size_t e = 0;
        for (size_t q = 0; q < rs; ++q) {
            rp[q] = (long long)e;
            const int i = nid[k][q];
            if (i < 0)
                continue;
            if (!I.dense)
                for (int64_t kk = m.row_ptr[i]; kk < m.row_ptr[i + 1]; ++kk, ++e) {
                    col[e] = pos[k][m.col[kk]];
                    w[e] = m.w[kk];
                }
            for (size_t j = 0; j < m.din; ++j)
                win[q * m.din + j] = m.W_in[(size_t)i * m.din + j];
            if (!I.dense)
                for (size_t oo = 0; oo < m.dout; ++oo)
                    wout[oo * rs + q] = m.W_out[oo * m.n + i];
        }
        rp[rs] = (long long)e;
        I.V = (double *)(A + o.V);
        I.tprev = (double *)(A + o.tp);
        I.ring = (double *)(A + o.ring);
        I.spk = (unsigned *)(A + o.spk);
        I.row_ptr = (const long long *)(A + o.rp);
        I.col = (const int *)(A + o.col);
        I.w = (const double *)(A + o.w);
        I.W_in = (const double *)(A + o.win);
        I.coef = (const double *)(A + o.coef);
        I.nid_of = (const int *)(A + o.nid);
        I.pos_of = (const int *)(A + o.pos);
        b->w_pos[k] = (double *)(A + o.wout);
        I.cmo = (const uint2 *)(A + o.cmo);
        I.cw = (const double *)(A + o.cw);
        I.nid_ro = I.dense ? (const int *)(A + o.nro) : I.nid_of;
        I.pos_ro = I.dense ? (const int *)(A + o.pro) : I.pos_of;
        if (I.dense)
            for (size_t q = 0; q < rs; ++q) {
                const int i = nid_ro[q];
                if (i >= 0)
                    for (size_t oo = 0; oo < m.dout; ++oo)
                        wout[oo * rs + q] = m.W_out[oo * m.n + i];
            }
        // synchronous copies: the staging vectors die at the end of this iteration
        bool ok = cudaMemcpy(A + o.rp, rp.data(), rp.size() * 8, cudaMemcpyHostToDevice) ==
                      cudaSuccess &&
                  cudaMemcpy(A + o.col, col.data(), col.size() * 4, cudaMemcpyHostToDevice) ==
                      cudaSuccess &&
                  cudaMemcpy(A + o.w, w.data(), w.size() * 8, cudaMemcpyHostToDevice) ==
                      cudaSuccess &&
                  cudaMemcpy(A + o.win, win.data(), win.size() * 8, cudaMemcpyHostToDevice) ==
                      cudaSuccess &&
                  cudaMemcpy(A + o.wout, wout.data(), wout.size() * 8, cudaMemcpyHostToDevice) ==
                      cudaSuccess &&
                  cudaMemcpy(A + o.nid, nid[k].data(), rs * 4, cudaMemcpyHostToDevice) ==
                      cudaSuccess &&
                  cudaMemcpy(A + o.pos, pos[k].data(), m.n * 4, cudaMemcpyHostToDevice) ==
                      cudaSuccess;
        if (ok && I.dense)
            ok = cudaMemcpy(A + o.nro, nid_ro.data(), rs * 4, cudaMemcpyHostToDevice) ==
                     cudaSuccess &&
                 cudaMemcpy(A + o.pro, pos_ro.data(), m.n * 4, cudaMemcpyHostToDevice) ==
                     cudaSuccess &&
                 cudaMemcpy(A + o.cmo, cmo.data(), cmo.size() * 8, cudaMemcpyHostToDevice) ==
                     cudaSuccess &&
                 cudaMemcpy(A + o.cw, cw.data(), cw.size() * 8, cudaMemcpyHostToDevice) ==
                     cudaSuccess;
        if (ok && I.ntype == SP_FLIF_GL)
            ok = cudaMemcpy(A + o.coef, m.coef, (size_t)I.L * 8, cudaMemcpyHostToDevice) ==
                 cudaSuccess;
        if (!ok) {
#pragma omp atomic write
            failed = 1;
        }
    }
    if (failed) {
        cudaGetLastError();
        sp_batch_destroy(b);
        return SP_EINTERNAL;
    }
    if (sp_cuda_malloc(&b->d_bar, (size_t)b->P * sizeof(unsigned long long)) != cudaSuccess ||
        sp_cuda_malloc(&b->d_err, 4 * sizeof(int)) != cudaSuccess ||
        sp_cuda_malloc(&b->d_inst, count * sizeof(BInst)) != cudaSuccess ||
        cudaMemset(b->d_err, 0, 4 * sizeof(int)) != cudaSuccess) {
        sp_batch_destroy(b);
        return SP_EALLOC;
    }
    *out = b;
    return SP_OK;
}

// Staging buffers and schedule for series lengths T (re-planned only when T
// or the need for states changes).
static int batch_prepare(sp_batch *b, const size_t *T, int want_phi)
{
    const size_t cnt = b->inst.size();
    bool same = b->T.size() == cnt && b->want_phi == want_phi;
    for (size_t k = 0; same && k < cnt; ++k)
        same = b->T[k] == (long long)T[k];
    if (same)
        return SP_OK;
    batch_free_run(b);
    b->T.assign(T, T + cnt);
    b->want_phi = want_phi;
    size_t u_total = 0, ras_total = 0, v_total = 0, phi_total = 0;
    for (size_t k = 0; k < cnt; ++k) {
        u_total += T[k] * b->inst[k].din;
        ras_total += T[k] * b->inst[k].nw;
        v_total += b->inst[k].n;
        phi_total += want_phi ? T[k] * b->inst[k].rs : 0;
    }
    b->u_total = u_total;
    b->ras_total = ras_total;
    b->v_total = v_total;
    b->phi_total = phi_total;
    BK(sp_cuda_malloc(&b->d_u, (u_total ? u_total : 1) * 8));
    BK(sp_cuda_malloc(&b->d_ras, (ras_total ? ras_total : 1) * 4));
    BK(sp_cuda_malloc(&b->d_ras_nat, (ras_total ? ras_total : 1) * 4));
    BK(sp_cuda_malloc(&b->d_vnat, v_total * 8));
    if (want_phi)
        BK(sp_cuda_malloc(&b->d_phi, (phi_total ? phi_total : 1) * 8));
    BK(cudaMallocHost(&b->h_u, (u_total ? u_total : 1) * 8));
    BK(cudaMallocHost(&b->h_ras, (ras_total ? ras_total : 1) * 4));
    BK(cudaMallocHost(&b->h_vnat, v_total * 8));
    size_t uo = 0, ro = 0, vo = 0, po = 0;
    for (size_t k = 0; k < cnt; ++k) {
        BInst &I = b->inst[k];
        I.T = (long long)T[k];
        I.u = b->d_u + uo;
        I.raster = b->d_ras + ro;
        I.raster_nat = b->d_ras_nat + ro;
        I.V_nat = b->d_vnat + vo;
        I.phi = want_phi ? b->d_phi + po : nullptr;
        uo += T[k] * I.din;
        ro += T[k] * I.nw;
        vo += I.n;
        po += want_phi ? T[k] * I.rs : 0;
    }
    plan(b, b->T);
    std::vector<int> sched;
    sched.insert(sched.end(), b->cta_group.begin(), b->cta_group.end());
    sched.insert(sched.end(), b->group_start.begin(), b->group_start.end());
    sched.insert(sched.end(), b->group_size.begin(), b->group_size.end());
    sched.insert(sched.end(), b->job_off.begin(), b->job_off.end());
    sched.insert(sched.end(), b->jobs.begin(), b->jobs.end());
    if (b->d_sched)
        sp_cuda_free(b->d_sched);
    b->d_sched = nullptr;
    BK(sp_cuda_malloc(&b->d_sched, sched.size() * sizeof(int)));
    BK(cudaMemcpy(b->d_sched, sched.data(), sched.size() * sizeof(int), cudaMemcpyHostToDevice));
    BK(cudaMemcpy(b->d_inst, b->inst.data(), cnt * sizeof(BInst), cudaMemcpyHostToDevice));
    return SP_OK;
}

// Device work of one run on b->stream (the sequence the graph captures).
static int batch_enqueue(sp_batch *b)
{
    const unsigned cnt = (unsigned)b->inst.size();
    BK(cudaMemcpyAsync(b->d_u, b->h_u, (b->u_total ? b->u_total : 1) * 8, cudaMemcpyHostToDevice,
                       b->stream));
    const dim3 rg(64, cnt);
    k_batch_reset<<<rg, 256, 0, b->stream>>>(b->d_inst);
    BK(cudaGetLastError());
    BK(cudaMemsetAsync(b->d_bar, 0, (size_t)b->P * sizeof(unsigned long long), b->stream));
    BParams p;
    const int P = b->P, G = b->ngroups;
    p.inst = b->d_inst;
    p.cta_group = b->d_sched;
    p.group_start = b->d_sched + P;
    p.group_size = b->d_sched + P + G;
    p.job_off = b->d_sched + P + 2 * G;
    p.jobs = b->d_sched + P + 3 * G + 1;
    p.bar = b->d_bar;
    p.err = b->d_err;
    p.lmax = b->lmax;
    p.max_nw = b->max_nw;
    p.list_cap = b->list_cap;
    void *args[] = {&p};
    BK(cudaLaunchCooperativeKernel((const void *)k_batch, dim3(P), dim3(kBatchThreads), args,
                                   b->smem, b->stream));
    k_batch_gather<<<rg, 256, 0, b->stream>>>(b->d_inst);
    BK(cudaGetLastError());
    BK(cudaMemcpyAsync(b->h_ras, b->d_ras_nat, (b->ras_total ? b->ras_total : 1) * 4,
                       cudaMemcpyDeviceToHost, b->stream));
    BK(cudaMemcpyAsync(b->h_vnat, b->d_vnat, b->v_total * 8, cudaMemcpyDeviceToHost, b->stream));
    return SP_OK;
}

// Stage inputs, replay (or capture) the graph, wait, check the error flag.
static int batch_simulate(sp_batch *b, const double *const *u, float *ms)
{
    const size_t cnt = b->inst.size();
    size_t uo = 0;
    for (size_t k = 0; k < cnt; ++k) {
        const size_t len = (size_t)b->T[k] * b->inst[k].din;
        if (u && u[k])
            memcpy(b->h_u + uo, u[k], len * 8);
        else
            memset(b->h_u + uo, 0, len * 8);
        uo += len;
    }
    if (b->graph_ok == 0) {
        cudaGraph_t g = nullptr;
        bool ok = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        if (ok) {
            const int r2 = batch_enqueue(b);
            ok = cudaStreamEndCapture(b->stream, &g) == cudaSuccess && r2 == SP_OK;
        }
        if (ok)
            ok = cudaGraphInstantiate(&b->graph, g, 0) == cudaSuccess;
        if (g)
            cudaGraphDestroy(g);
        cudaGetLastError();
        b->graph_ok = ok ? 1 : -1;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    BK(cudaEventCreate(&e0));
    BK(cudaEventCreate(&e1));
    BK(cudaEventRecord(e0, b->stream));
    int rc = SP_OK;
    if (b->graph_ok == 1) {
        if (cudaGraphLaunch(b->graph, b->stream) != cudaSuccess)
            rc = SP_EINTERNAL;
    } else {
        rc = batch_enqueue(b);
    }
    cudaEventRecord(e1, b->stream);
    if (cudaStreamSynchronize(b->stream) != cudaSuccess)
        rc = SP_EINTERNAL;
    if (!rc && ms)
        cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc)
        return rc;
    b->runs++;
    int herr[2] = {0, 0};
    BK(cudaMemcpy(herr, b->d_err, sizeof(herr), cudaMemcpyDeviceToHost));
    if (herr[0] != 0) {
        fprintf(stderr, "spires: batch kernel error %d at micro-step %d\n", herr[0], herr[1]);
        cudaMemset(b->d_err, 0, 4 * sizeof(int));
        return SP_EINTERNAL;
    }
    return SP_OK;
}

extern "C" int sp_batch_run(sp_batch *b, const double *const *u, const size_t *T,
                            uint32_t *const *raster, double *const *final_state,
                            double *elapsed_ms)
{
    int rc = batch_prepare(b, T, 0);
    if (rc)
        return rc;
    float ms = 0.f;
    rc = batch_simulate(b, u, &ms);
    if (rc)
        return rc;
    if (elapsed_ms)
        *elapsed_ms = ms;
    size_t ro = 0, vo = 0;
    for (size_t k = 0; k < b->inst.size(); ++k) {
        const size_t len = (size_t)b->T[k] * b->inst[k].nw;
        if (raster && raster[k])
            memcpy(raster[k], b->h_ras + ro, len * 4);
        if (final_state && final_state[k])
            memcpy(final_state[k], b->h_vnat + vo, (size_t)b->inst[k].n * 8);
        ro += len;
        vo += b->inst[k].n;
    }
    return SP_OK;
}

// Readouts of one instance over its recorded states, with the single path's
// layout and reduction (so the bits match spires_run): column-block
// instances first move their states from neuron order to that layout.
static int batch_readout(sp_batch *b, const BInst &I, const double *phi, size_t T, int dout,
                         double *Y)
{
    if (!I.dense)
        return sp_launch_readout(b->stream, b->w_pos[&I - b->inst.data()], phi, I.rs, T, dout, Y);
    double *tmp = nullptr;
    if (sp_cuda_malloc_async(&tmp, (T ? T : 1) * (size_t)I.rs * sizeof(double), b->stream) !=
        cudaSuccess) {
        cudaGetLastError();
        return SP_EALLOC;
    }
    const size_t total = T * (size_t)I.rs;
    const unsigned blocks = (unsigned)std::min<size_t>((total + 255) / 256, 16384);
    k_rows_to_layout<<<blocks ? blocks : 1, 256, 0, b->stream>>>(phi, I.rs, I.nid_ro, T, tmp);
    int rc = cudaGetLastError() == cudaSuccess ? SP_OK : SP_EINTERNAL;
    if (!rc)
        rc = sp_launch_readout(b->stream, b->w_pos[&I - b->inst.data()], tmp, I.rs, T, dout, Y);
    sp_cuda_free_async(tmp, b->stream);
    return rc;
}

// Ridge readouts of every instance from one batched simulation: states of
// all instances recorded in one launch, then per instance the FP64 ridge of
// the single-reservoir path (Gram + Cholesky + refinement) on its states.
extern "C" int sp_batch_train_ridge(sp_batch *b, const double *const *u, const double *const *y,
                                    const size_t *T, const double *lambda,
                                    const sp_ridge_opts *o, double *const *w_out,
                                    double *elapsed_ms)
{
    auto t0 = std::chrono::steady_clock::now();
    int rc = batch_prepare(b, T, 1);
    if (rc)
        return rc;
    rc = batch_simulate(b, u, nullptr);
    if (rc)
        return rc;
    size_t max_tn = 1, max_ty = 1, max_wn = 1;
    for (size_t k = 0; k < b->inst.size(); ++k) {
        max_tn = std::max(max_tn, T[k] * (size_t)b->inst[k].n);
        max_ty = std::max(max_ty, T[k] * b->models[k].dout);
        max_wn = std::max(max_wn, (size_t)b->inst[k].n * b->models[k].dout);
    }
    double *nat = nullptr, *Y = nullptr, *W = nullptr;
    sp_ridge_ws *ws = sp_ridge_ws_new();  // one set of solver buffers for every instance
    auto cleanup = [&]() {
        cudaStreamSynchronize(b->stream);
        sp_ridge_ws_free(ws);
        if (nat)
            sp_cuda_free(nat);
        if (Y)
            sp_cuda_free(Y);
        if (W)
            sp_cuda_free(W);
    };
    if (sp_cuda_malloc(&nat, max_tn * 8) != cudaSuccess || sp_cuda_malloc(&Y, max_ty * 8) != cudaSuccess ||
        sp_cuda_malloc(&W, max_wn * 8) != cudaSuccess) {
        cudaGetLastError();
        cleanup();
        return SP_EALLOC;
    }
    size_t po = 0;
    for (size_t k = 0; k < b->inst.size() && !rc; ++k) {
        const BInst &I = b->inst[k];
        const int dout = (int)b->models[k].dout;
        const double *phi = b->d_phi + po;
        po += T[k] * I.rs;
        if (dout == 0)
            continue;
        if (cudaMemcpyAsync(Y, y[k], T[k] * dout * 8, cudaMemcpyHostToDevice, b->stream) !=
            cudaSuccess) {
            rc = SP_EINTERNAL;
            break;
        }
        rc = sp_launch_gather_rows(b->stream, phi, I.rs, I.pos_of, I.n, T[k], nat);
        if (rc)
            break;
        sp_ridge_report rep;
        memset(&rep, 0, sizeof(rep));
        rc = sp_ridge_phi_ws(b->stream, nat, I.n, T[k], Y, dout, lambda[k], o, &rep, W, ws);
        if (rc == SP_RIDGE_SINGULAR) {
            // singular: W_out of this instance stays as it was (dgesv failure)
            rc = SP_OK;
            if (w_out && w_out[k]) {
                rc = sp_launch_gather_rows(b->stream, b->w_pos[k], I.rs, I.pos_ro, I.n,
                                           (size_t)dout, W);
                if (!rc && cudaMemcpy(w_out[k], W, (size_t)dout * I.n * 8,
                                      cudaMemcpyDeviceToHost) != cudaSuccess)
                    rc = SP_EINTERNAL;
            }
            continue;
        }
        if (rc)
            break;
        rc = sp_launch_wout_to_pos(b->stream, W, I.nid_ro, I.n, I.rs, dout, b->w_pos[k]);
        if (!rc && w_out && w_out[k] &&
            cudaMemcpyAsync(w_out[k], W, (size_t)dout * I.n * 8, cudaMemcpyDeviceToHost,
                            b->stream) != cudaSuccess)
            rc = SP_EINTERNAL;
        if (!rc && cudaStreamSynchronize(b->stream) != cudaSuccess)
            rc = SP_EINTERNAL;
    }
    cleanup();
    if (elapsed_ms)
        *elapsed_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

// Readouts of every instance over its series from reset, with its current
// W_out: y[k] is T[k] x dout, the same arithmetic as spires_run.
extern "C" int sp_batch_predict(sp_batch *b, const double *const *u, const size_t *T,
                                double *const *y, double *elapsed_ms)
{
    auto t0 = std::chrono::steady_clock::now();
    int rc = batch_prepare(b, T, 1);
    if (rc)
        return rc;
    rc = batch_simulate(b, u, nullptr);
    if (rc)
        return rc;
    size_t max_ty = 1;
    for (size_t k = 0; k < b->inst.size(); ++k)
        max_ty = std::max(max_ty, T[k] * b->models[k].dout);
    double *Y = nullptr;
    BK(sp_cuda_malloc(&Y, max_ty * 8));
    size_t po = 0;
    for (size_t k = 0; k < b->inst.size() && !rc; ++k) {
        const BInst &I = b->inst[k];
        const int dout = (int)b->models[k].dout;
        const double *phi = b->d_phi + po;
        po += T[k] * I.rs;
        if (dout == 0 || !y || !y[k])
            continue;
        rc = batch_readout(b, I, phi, T[k], dout, Y);
        if (!rc && cudaMemcpyAsync(y[k], Y, T[k] * dout * 8, cudaMemcpyDeviceToHost, b->stream) !=
                       cudaSuccess)
            rc = SP_EINTERNAL;
        if (!rc && cudaStreamSynchronize(b->stream) != cudaSuccess)
            rc = SP_EINTERNAL;
    }
    cudaStreamSynchronize(b->stream);
    sp_cuda_free(Y);
    if (elapsed_ms)
        *elapsed_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

// One simulation per instance serves both the fit and the score: states of
// T[k] steps are recorded, the ridge uses rows [washout, T_fit[k]) and the
// fitted readout is applied to every row, y_out[k] being T[k] x dout.
extern "C" int sp_batch_fit_predict(sp_batch *b, const double *const *u, const double *const *y,
                                    const size_t *T, const size_t *T_fit, const double *lambda,
                                    const sp_ridge_opts *o, double *const *y_out,
                                    double *const *w_out, double *elapsed_ms)
{
    auto t0 = std::chrono::steady_clock::now();
    int rc = batch_prepare(b, T, 1);
    if (rc)
        return rc;
    rc = batch_simulate(b, u, nullptr);
    if (rc)
        return rc;
    size_t max_tn = 1, max_ty = 1, max_wn = 1;
    for (size_t k = 0; k < b->inst.size(); ++k) {
        max_tn = std::max(max_tn, T_fit[k] * (size_t)b->inst[k].n);
        max_ty = std::max(max_ty, T[k] * b->models[k].dout);
        max_wn = std::max(max_wn, (size_t)b->inst[k].n * b->models[k].dout);
    }
    double *nat = nullptr, *Y = nullptr, *W = nullptr;
    if (sp_cuda_malloc(&nat, max_tn * 8) != cudaSuccess || sp_cuda_malloc(&Y, max_ty * 8) != cudaSuccess ||
        sp_cuda_malloc(&W, max_wn * 8) != cudaSuccess) {
        cudaGetLastError();
        if (nat)
            sp_cuda_free(nat);
        if (Y)
            sp_cuda_free(Y);
        return SP_EALLOC;
    }
    size_t po = 0;
    sp_ridge_ws *ws = sp_ridge_ws_new();  // one set of solver buffers for every instance
    for (size_t k = 0; k < b->inst.size() && !rc; ++k) {
        const BInst &I = b->inst[k];
        const int dout = (int)b->models[k].dout;
        const double *phi = b->d_phi + po;
        po += T[k] * I.rs;
        if (dout == 0)
            continue;
        if (cudaMemcpyAsync(Y, y[k], T_fit[k] * dout * 8, cudaMemcpyHostToDevice, b->stream) !=
            cudaSuccess) {
            rc = SP_EINTERNAL;
            break;
        }
        rc = sp_launch_gather_rows(b->stream, phi, I.rs, I.pos_of, I.n, T_fit[k], nat);
        if (rc)
            break;
        sp_ridge_report rep;
        memset(&rep, 0, sizeof(rep));
        rc = sp_ridge_phi_ws(b->stream, nat, I.n, T_fit[k], Y, dout, lambda[k], o, &rep, W, ws);
        if (rc == SP_RIDGE_SINGULAR) {
            rc = SP_OK; /* this instance keeps its previous W_out */
        } else if (!rc) {
            rc = sp_launch_wout_to_pos(b->stream, W, I.nid_ro, I.n, I.rs, dout, b->w_pos[k]);
            if (!rc && w_out && w_out[k] &&
                cudaMemcpyAsync(w_out[k], W, (size_t)dout * I.n * 8, cudaMemcpyDeviceToHost,
                                b->stream) != cudaSuccess)
                rc = SP_EINTERNAL;
        }
        if (rc)
            break;
        rc = batch_readout(b, I, phi, T[k], dout, Y);
        if (!rc && y_out && y_out[k] &&
            cudaMemcpyAsync(y_out[k], Y, T[k] * dout * 8, cudaMemcpyDeviceToHost, b->stream) !=
                cudaSuccess)
            rc = SP_EINTERNAL;
        if (!rc && cudaStreamSynchronize(b->stream) != cudaSuccess)
            rc = SP_EINTERNAL;
        if (rc && getenv("SPIRES_DEBUG"))
            fprintf(stderr, "spires: batch fit of instance %zu (n %d, rows %zu, washout %zu) failed: %d\n",
                    k, I.n, T_fit[k], o->washout, rc);
    }
    cudaStreamSynchronize(b->stream);
    sp_ridge_ws_free(ws);
    sp_cuda_free(nat);
    sp_cuda_free(Y);
    sp_cuda_free(W);
    if (elapsed_ms)
        *elapsed_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

// Autotuner: times every schedule family on a grid of full occupancy and
// on one CTA per SM, with the caller's series (the run starts every instance
// from reset, so no state needs saving), keeps the fastest and returns its
// device time. Later runs plan with the chosen family and grid.
extern "C" int sp_batch_autotune(sp_batch *b, const double *const *u, const size_t *T,
                                 int *best_mode, int *best_ctas, double *best_ms)
{
    std::vector<int> grids = {b->P_max};
    if (b->P_max > b->num_sms)
        grids.push_back(b->num_sms);
    const int mode0 = b->plan_mode, P0 = b->P;
    int bm = mode0, bp = P0;
    float best = 3.4e38f;
    for (int P : grids) {
        bool fits = true;
        for (const BInst &I : b->inst)
            fits = fits && min_ctas(I) <= P;
        if (!fits)
            continue;
        for (int mode = 0; mode < 4; ++mode) {
            b->P = P;
            b->plan_mode = mode;
            b->T.clear();  // re-plan and re-capture
            int rc = batch_prepare(b, T, 0);
            float ms = 0.f;
            if (!rc)
                rc = batch_simulate(b, u, &ms);
            if (rc) {
                b->P = P0;
                b->plan_mode = mode0;
                b->T.clear();
                return rc;
            }
            if (ms < best) {
                best = ms;
                bm = mode;
                bp = P;
            }
        }
    }
    b->P = bp;
    b->plan_mode = bm;
    b->T.clear();
    if (best_mode)
        *best_mode = bm;
    if (best_ctas)
        *best_ctas = bp;
    if (best_ms)
        *best_ms = best;
    return SP_OK;
}

extern "C" int sp_batch_info(const sp_batch *b, int *ctas, int *groups, int *graph)
{
    if (ctas)
        *ctas = b->P;
    if (groups)
        *groups = b->ngroups;
    if (graph)
        *graph = b->graph_ok;
    return SP_OK;
}

#ifdef SP_PHASE_STAMPS
extern "C" __attribute__((visibility("default"))) int spires_dbg_batch_job_stamps(void *host,
                                                                                 size_t bytes)
{
    if (bytes < sizeof(g_sp_jobstamps))
        return -1;
    if (cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpyFromSymbol(host, g_sp_jobstamps, sizeof(g_sp_jobstamps)) != cudaSuccess)
        return -1;
    // cleared after each read, so the next read holds only the runs since
    void *sym = nullptr;
    if (cudaGetSymbolAddress(&sym, g_sp_jobstamps) != cudaSuccess ||
        cudaMemset(sym, 0, sizeof(g_sp_jobstamps)) != cudaSuccess ||
        cudaDeviceSynchronize() != cudaSuccess)
        return -1;
    return 0;
}
#endif
