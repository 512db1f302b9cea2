// sp_step_kernel.cuh -- the persistent reservoir step kernel (all neuron and
// synapse models), included by dev_reservoir.cu.
//
// Launch: a cooperative grid of G CTAs; CTA b owns the whole warps
// [b*nw/G, (b+1)*nw/G) of neurons (nw = ceil(n/32)); a consumer thread owns
// one neuron and keeps its state in registers for the whole launch.
//
// Variant 0: the FLIF_GL history is summed with direct loads from the
//   time-major ring (each lag is one coalesced row segment).
// Variant 1 (FLIF_GL only): one extra producer warp streams the ring rows of
//   the CTA's neuron range into a multi-stage shared-memory pipeline with
//   cp.async.bulk (bulk-copy TMA) on mbarriers; the consumers read lags from
//   shared memory. The producer runs up to one step ahead of the consumers:
//   the rows of step g are the states of steps <= g-2 (lag 1 is the register
//   copy of the previous state), so they only wait for step g-2 to finish.
//   Lags 2..33 are the thread's own last 32 states, kept in a register shift
//   register, so the producer streams lags 34.. only (3 % fewer ring bytes per
//   step at L = 1024) and the sum of a step starts as soon as its lag 1 exists.
//   The grid is sized so that each CTA streams about the same number of ring
//   columns (balanced layout, dev_reservoir.cu), and the CTA's CSR slice sits
//   in shared memory for the launch, so the row pass after each grid barrier
//   reads no global memory but the spike words. A gather warp watches the
//   other CTAs' arrival flags and copies their spike words into a
//   double-buffered shared array while the consumers are still summing.
//   A ring larger than the L2 is read with cache hints: the oldest l2_pin
//   lags of a step are loaded with evict-last priority and stay L2-resident
//   from step to step (each row joins them once, when it reaches lag
//   L - l2_pin), the younger lags stream through with evict-first, so the
//   DRAM reads come first in every step and run on through the serial phase.
//
// Per micro-step (both variants), with a split-phase grid barrier:
//   history sum of step g      (overlaps the barrier wait)
//   wait barrier g             (spike words / eff of step g-1 visible)
//   recurrent input            SIMPLE: warp-cooperative walk over the warp's
//                              CSR edges, ballot of spiking presynaptic bits,
//                              owner lane adds the weights in ascending edge
//                              order; others: warp-cooperative walk, one
//                              term per edge, owner lane adds in edge order
//   neuron update, ring write, ballot -> spike word of step g
//   synapse prepare for g+1 (own spike), publish, arrive barrier g+1
#pragma once
#include <cuda.h>
#include "sp_kernels.cuh"
#include "sp_model.h"

namespace sp {

struct KP {
    int n, nwords, din, micro, G, n_macro, phase0;
    int rs;         // ring row stride in doubles (multiple of 32)
    int warps;      // consumer warps per CTA
    int R, NST;     // variant 1: ring rows per stage, stages
    int BW, NBX;    // variant 1: box width (neurons) and boxes side by side per stage
    int bal;        // balanced layout: CTA b's active positions are the first
                    // n / G (+1 for b < n % G) of its range, the rest holes
    int RB;         // variant 1: rows per box = min(R, L)
    int coef_smem;  // variant 1: coefficient table staged in shared memory
    int csr_cap;    // SIMPLE synapse: edges of the CTA's CSR slice kept in shared
                    // memory for the launch (0: rows are walked in global memory)
    const int *nid_of;  // neuron at each position, -1 for an empty lane
    long long step0, syn_step0;
    double a, b, c, d, e, f, g, h, ci, cj, ck, cl, dt;
    int L, det_refr, diff_sto;
    const double *coef;
    double *V, *tprev, *ring;
    int *cap_pos;
    long long *refr_until;
    unsigned long long *rng;
    unsigned *spk;
    const long long *row_ptr;
    const int *col;
    const double *w;
    double *eff;
    double psc_decay, psc_omd;
    double *trace;
    const double *edge_decay, *edge_omd;
    double *edge_trace;
    int Ls;
    const double *scoef;
    double s_dta, s_tau;
    double *Iring;
    int Nc;
    const double *mx_decay, *mx_omd, *mx_c;
    double *mx_tr;
    const double *W_in;
    double gamma;
    const double *u;
    double *phi;
    unsigned *raster;
    unsigned long long *bar;  // grid-barrier arrival counter (64-bit: never wraps)
    // arrival flags, one per CTA on its own 128-byte line: CTA c stores b + 1
    // once its spike words and drive of micro-step b - 1 are published
    unsigned long long *flags;
    int *err;                 // [0] error code, [1] / [2] low / high word of the micro-step
    unsigned long long tmo;   // limit of every wait, ns
    // one-shot test hook: CTA hold_cta does not arrive at the barrier that
    // opens micro-step hold_b (-1: none), so every wait on it runs out
    int hold_cta;
    long long hold_b;
    // variant 1: the oldest l2_pin lags of every step are read with L2
    // evict-last priority, younger ones and the ring writes with evict-first
    // (0: no hints)
    int l2_pin;
    // variant 1: 2-D tiled map of the ring [L rows][rs columns] of doubles,
    // box = BW columns x R rows
    alignas(64) CUtensorMap tmap;
};

// ------------------------------------------------------------ PTX helpers
__device__ __forceinline__ unsigned smem_u32(const void *p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void named_sync(int n)
{
    asm volatile("bar.sync 1, %0;" ::"r"(n) : "memory");
}
__device__ __forceinline__ void mbar_init(unsigned long long *b, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ bool mbar_test(unsigned long long *b, unsigned parity)
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
// read-only load that does not allocate in L1 (per-step input weights must not
// evict the coefficient table and the CSR slice)
__device__ __forceinline__ double ldg_na(const double *ptr)
{
    double v;
    asm volatile("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(ptr));
    return v;
}

// 2-D tiled bulk-tensor load of one box at (x = column, y = row); no multicast.
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y,
                                            unsigned long long *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}
// L2 eviction-priority policies for the cache-hinted ring loads and stores:
// evict-last for the slots kept resident, evict-first for the streamed ones
__device__ __forceinline__ unsigned long long l2_policy(bool keep)
{
    unsigned long long pol;
    if (keep)
        asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    else
        asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ void tma_load_2d_hint(void *dst, const CUtensorMap *map, int x, int y,
                                                 unsigned long long *bar, unsigned long long pol)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        ".L2::cache_hint [%0], [%1, {%2, %3}], [%4], %5;" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(smem_u32(bar)),
        "l"(pol)
        : "memory");
}
__device__ __forceinline__ void st_hint_f64(double *ptr, double v, unsigned long long pol)
{
    asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(ptr), "d"(v), "l"(pol)
                 : "memory");
}
__device__ __forceinline__ void st_release_cta(volatile int *ptr, int v)
{
    asm volatile("st.release.cta.shared::cta.s32 [%0], %1;" ::"r"(smem_u32((const void *)ptr)),
                 "r"(v)
                 : "memory");
}
__device__ __forceinline__ int ld_acquire_cta(volatile int *ptr)
{
    int v;
    asm volatile("ld.acquire.cta.shared::cta.s32 %0, [%1];"
                 : "=r"(v)
                 : "r"(smem_u32((const void *)ptr))
                 : "memory");
    return v;
}
__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async;" ::: "memory");
}

// Bounded mbarrier wait; false on timeout or when the launch is aborting.
__device__ __forceinline__ void record_err(int *err, int code, long long step)
{
    if (atomicCAS(err, kErrNone, code) == kErrNone) {
        err[1] = (int)(unsigned)(unsigned long long)step;
        err[2] = (int)(unsigned)((unsigned long long)step >> 32);
    }
}

__device__ __forceinline__ bool mbar_wait(unsigned long long *b, unsigned parity,
                                          volatile int *s_abort, int *err,
                                          unsigned long long tmo, long long step)
{
    if (mbar_test(b, parity))
        return true;
    unsigned long long t0 = globaltimer_ns();
    unsigned polls = 0;
    while (!mbar_test(b, parity)) {
        if ((++polls & 63u) == 0) {
            if (*s_abort || ld_volatile_i32(err) != kErrNone)
                return false;
            if (globaltimer_ns() - t0 > tmo) {
                record_err(err, kErrBarrierTimeout, step);
                *s_abort = 1;
                return false;
            }
        }
    }
    return true;
}

// SIMPLE synapse, one warp: recurrent input of rows [row0, row0 + nv) for the
// lane that owns row row0 + lane. Edges are scanned 32 at a time; spiking
// presynaptic columns are found by a ballot over the spike bits and each
// weight is added by the owner lane of its row in ascending edge order, i.e.
// exactly the non-zero terms of csr_row_dot (src/sparse.c:68-76) in order.
__device__ __forceinline__ double rowpass_simple_warp(const long long *__restrict__ row_ptr,
                                                      const int *__restrict__ col,
                                                      const double *__restrict__ w,
                                                      const unsigned *s_spk, int row0, int nv,
                                                      int lane)
{
    const long long e0 = __ldg(row_ptr + row0);
    const long long e1 = __ldg(row_ptr + row0 + nv);
    const long long my_end = (lane < nv) ? __ldg(row_ptr + row0 + lane + 1) : e1;
    double acc = 0.0;
    // next chunk's column index and weight are loaded one chunk ahead
    int cn = -1;
    double wn = 0.0;
    if (e0 + lane < e1) {
        cn = __ldg(col + e0 + lane);
        wn = __ldg(w + e0 + lane);
    }
    for (long long base = e0; base < e1; base += 32) {
        const int c = cn;
        const double wv = wn;
        const long long nx = base + 32 + lane;
        cn = -1;
        if (nx < e1) {
            cn = __ldg(col + nx);
            wn = __ldg(w + nx);
        }
        const bool s = c >= 0 && ((s_spk[c >> 5] >> (c & 31)) & 1u);
        unsigned m = __ballot_sync(kFull, s);
        while (m) {
            const int bpos = __ffs(m) - 1;
            m &= m - 1;
            const long long eb = base + bpos;
            const double wb = __shfl_sync(kFull, wv, bpos);
            const unsigned owner = __ballot_sync(kFull, my_end > eb);
            if (lane == __ffs(owner) - 1)
                acc = add(acc, wb);
        }
    }
    return acc;
}

// Per-phase timing of the last kSpStampSteps micro-steps of a launch
// (compiled in only with -DSP_PHASE_STAMPS): thread 0 of each CTA records the
// global timer at the phase boundaries of every step into g_sp_stamps
// [cta][step][phase]; spires_dbg_phase_stamps (dev_reservoir.cu) copies them
// out. Phases: 0 step start, 1 history summed, 2 barrier passed, 3 spike
// words staged, 4 row pass done (warp 0), 5 update and spike word done,
// 6 arrival made; 7 the producer issued the step's first stage.
#ifdef SP_PHASE_STAMPS
constexpr int kSpStampCtas = 160, kSpStampSteps = 32, kSpStampPhases = 8;
__device__ unsigned long long g_sp_stamps[kSpStampCtas * kSpStampSteps * kSpStampPhases];
#define SP_STAMP(cond, b, B, ph)                                                             \
    do {                                                                                    \
        if ((cond) && blockIdx.x < kSpStampCtas && (b) >= (B)-kSpStampSteps)                \
            g_sp_stamps[((size_t)blockIdx.x * kSpStampSteps + ((b) - ((B)-kSpStampSteps))) * \
                            kSpStampPhases +                                                \
                        (ph)] = globaltimer_ns();                                           \
    } while (0)
#else
#define SP_STAMP(cond, b, B, ph) \
    do {                         \
    } while (0)
#endif

// Synapses whose drive is not a spike bit (PSC and fractional: every edge
// carries a term), one warp: rows [row0, row0 + 32), lane r owns row row0 + r.
// The warp's contiguous edge range is taken 32 edges at a time, each lane
// forming one edge's term in parallel -- w_k * eff[col_k], or for
// PSC_HETEROGENEOUS the updated edge trace times w_k -- and the owner lane
// of each edge's row adds the terms in ascending edge order, the order of the
// reference's per-row loop (src/synapses/psc_heterogeneous.c:124-139,
// src/synapse.c:90-105), so the sums are the same bits as a per-row walk.
template <int ST>
__device__ __forceinline__ double rowpass_terms_warp(const KP &p, const double *ef,
                                                     const unsigned *s_spk, int row0, int lane)
{
    const long long e0 = __ldg(p.row_ptr + row0), e1 = __ldg(p.row_ptr + row0 + 32);
    const long long my_start = __ldg(p.row_ptr + row0 + lane);
    const long long my_end = __ldg(p.row_ptr + row0 + lane + 1);
    auto term_of = [&](long long k) -> double {
        if (k >= e1)
            return 0.0;
        const int c = __ldg(p.col + k);
        if (ST == SP_SYN_PSC_HET) {
            const double sv = ((s_spk[c >> 5] >> (c & 31)) & 1u) ? 1.0 : 0.0;
            const double tr = add(mul(p.edge_trace[k], __ldg(p.edge_decay + k)),
                                  mul(__ldg(p.edge_omd + k), sv));
            p.edge_trace[k] = tr;
            return mul(__ldg(p.w + k), tr);
        }
        return mul(__ldg(p.w + k), __ldcg(ef + c));
    };
    double acc = 0.0;
    // 4 chunks of 32 edges at a time: their loads in flight together, then
    // each chunk's terms added by the owner lanes in ascending edge order
    for (long long base = e0; base < e1; base += 4 * 32) {
        double t[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
            t[u] = term_of(base + 32 * u + lane);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const long long cb = base + 32 * u;
            if (cb >= e1)
                break;
            const int cnt = e1 - cb < 32 ? (int)(e1 - cb) : 32;
            for (int j = 0; j < cnt; ++j) {
                const double v = __shfl_sync(kFull, t[u], j);
                const long long eb = cb + j;
                if (eb >= my_start && eb < my_end)
                    acc = add(acc, v);
            }
        }
    }
    return acc;
}

// The same walk over the CTA's CSR slice in shared memory: rp = row offsets
// relative to the slice (rows of the CTA in position order), col = column
// positions, w = weights. Same terms, same order.
__device__ __forceinline__ double rowpass_simple_smem(const int *rp, const int *col,
                                                      const double *w, const unsigned *s_spk,
                                                      int row0, int lane)
{
    const int e0 = rp[row0], e1 = rp[row0 + 32];
    const int my_end = rp[row0 + lane + 1];
    double acc = 0.0;
    for (int base = e0; base < e1; base += 32) {
        const int e = base + lane;
        int c = -1;
        double wv = 0.0;
        if (e < e1) {
            c = col[e];
            wv = w[e];
        }
        const bool s = c >= 0 && ((s_spk[c >> 5] >> (c & 31)) & 1u);
        unsigned m = __ballot_sync(kFull, s);
        while (m) {
            const int bpos = __ffs(m) - 1;
            m &= m - 1;
            const int eb = base + bpos;
            const double wb = __shfl_sync(kFull, wv, bpos);
            const unsigned owner = __ballot_sync(kFull, my_end > eb);
            if (lane == __ffs(owner) - 1)
                acc = add(acc, wb);
        }
    }
    return acc;
}

template <int R>
__device__ __forceinline__ double stage_sum(double hist, const double *coef_k, const double *buf,
                                            int bw)
{
    double c[R], v[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
        c[j] = coef_k[j];
        v[j] = buf[(size_t)(R - 1 - j) * bw];
    }
#pragma unroll
    for (int j = 0; j < R; ++j)
        hist = add(hist, mul(c[j], v[j]));
    return hist;
}

// Variant 1 runs at most kPipeWarps consumer warps + 1 producer warp per CTA,
// which leaves registers for a stage of lags in flight and the register lags
// per thread.
constexpr int kPipeWarps = 8;

template <int VAR>
struct Bounds {
    static constexpr int threads = VAR == 1 ? 32 * (kPipeWarps + 2) : 1024;
};

// Variant 1 keeps lags 2..kRegLags+1 of its own neuron in registers: they are
// the thread's own last states, so they are neither written to nor read back
// from the ring for the sum, and the producer streams lags kRegLags+2.. only.
constexpr int kRegLags = 32;
constexpr int kFlagStride = 16;  // u64 per CTA arrival flag (one 128-byte line)

template <int NT, int ST, int VAR>
__global__ void __launch_bounds__(Bounds<VAR>::threads, 1) k_run(const __grid_constant__ KP p)
{
    constexpr int RL = (VAR == 1 && NT == SP_FLIF_GL) ? kRegLags : 0;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int s_flag;
    __shared__ volatile int s_abort;
    __shared__ volatile int s_done;
    __shared__ volatile int s_gather;  // variant 1: barriers whose words are staged

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int NC = 32 * p.warps;  // consumer threads
    const int wb0 = (int)(((long long)blockIdx.x * p.nwords) / p.G);
    const int wb1 = (int)(((long long)(blockIdx.x + 1) * p.nwords) / p.G);
    const int L = p.L;
    const long long B = (long long)p.n_macro * p.micro;

    // spike words of the barrier: one buffer, or two (variant 1: the gather
    // warp fills barrier b + 1's while the row pass reads barrier b's)
    const size_t spk_one = (((size_t)p.nwords * 4) + 127) & ~(size_t)127;
    unsigned *s_spkb = (unsigned *)smem;
    const size_t spk_bytes0 = (VAR == 1 ? 2 : 1) * spk_one;
    // CSR slice (SIMPLE synapse), between the spike words and the rest
    double *s_csr_w = (double *)(smem + spk_bytes0);
    const size_t csr_w_bytes = ((size_t)p.csr_cap * 8 + 127) / 128 * 128;
    int *s_csr_col = (int *)(smem + spk_bytes0 + csr_w_bytes);
    const size_t csr_c_bytes = ((size_t)p.csr_cap * 4 + 127) / 128 * 128;
    int *s_csr_rp = (int *)(smem + spk_bytes0 + csr_w_bytes + csr_c_bytes);
    const size_t csr_bytes =
        p.csr_cap > 0 ? csr_w_bytes + csr_c_bytes +
                            (((size_t)32 * p.warps + 1) * 4 + 127) / 128 * 128
                      : 0;
    const size_t spk_bytes = spk_bytes0 + csr_bytes;
    const size_t coef_bytes = p.coef_smem ? (((size_t)L * 8) + 127) & ~(size_t)127 : 0;
    double *s_coef = (double *)(smem + spk_bytes);
    double *s_stage = (double *)(smem + spk_bytes + coef_bytes);
    const size_t STAGE = (size_t)p.NBX * p.R * p.BW;  // doubles per stage
    unsigned long long *full = (unsigned long long *)(smem + spk_bytes + coef_bytes +
                                                      (size_t)p.NST * STAGE * sizeof(double));
    unsigned long long *empty = full + p.NST;
    const int lo = wb0 * 32;
    const int S_b = 32 * (wb1 - wb0);

    if (tid == 0) {
        s_abort = 0;
        s_done = 0;
        s_gather = 0;
    }
    if (VAR == 1 && p.coef_smem)
        for (int k = tid; k < L; k += blockDim.x)
            s_coef[k] = p.coef[k];
    if (ST == SP_SYN_SIMPLE && p.csr_cap > 0) {
        const long long e_lo = __ldg(p.row_ptr + lo);
        const int ne = (int)(__ldg(p.row_ptr + lo + S_b) - e_lo);  // <= csr_cap
        for (int k = tid; k < ne; k += blockDim.x) {
            s_csr_col[k] = __ldg(p.col + e_lo + k);
            s_csr_w[k] = __ldg(p.w + e_lo + k);
        }
        for (int q = tid; q <= S_b; q += blockDim.x)
            s_csr_rp[q] = (int)(__ldg(p.row_ptr + lo + q) - e_lo);
    }
    if (VAR == 1) {
        if (tid == 0) {
            for (int s = 0; s < p.NST; ++s) {
                mbar_init(&full[s], 1);
                mbar_init(&empty[s], p.warps);
            }
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
    }
    __syncthreads();

    // ------------------------------------------------------------ producer
    // ------------------------------------------------------------ gatherer
    // Variant 1, one warp: for barrier b it watches the arrival flags of all
    // CTAs (lane l: CTAs l, l + 32, ...), copies each CTA's spike words into
    // s_spkb[b & 1] as soon as that CTA's flag is up, and announces the
    // barrier in s_gather -- while the consumers are still summing history.
    // Buffer b & 1 is free by then: a flag can reach b + 1 only after this
    // CTA's arrival at barrier b - 1, which follows its row pass of b - 2.
    if (VAR == 1 && tid >= NC + 32) {
        constexpr bool kWords = ST == SP_SYN_SIMPLE || ST == SP_SYN_PSC_HET;
        if (p.G <= 1)
            return;
        for (long long b = 0; b < B; ++b) {
            const unsigned long long want = (unsigned long long)(b + 1);
            const int curb = p.phase0 ^ (int)(b & 1);
            unsigned *dst = s_spkb + (size_t)(b & 1) * (spk_one / 4);
            bool ok = true;
            for (int c = lane; c < p.G && ok; c += 32) {
                const unsigned long long *f = p.flags + (size_t)c * kFlagStride;
                if (ld_volatile_u64(f) < want) {
                    const unsigned long long t0 = globaltimer_ns();
                    unsigned long long polls = 0;
                    while (ld_volatile_u64(f) < want) {
                        if ((++polls & 255ull) == 0) {
                            if (s_abort || ld_volatile_i32(p.err) != kErrNone) {
                                ok = false;
                                break;
                            }
                            if (globaltimer_ns() - t0 > p.tmo || polls > kBarrierMaxPolls) {
                                record_err(p.err, kErrBarrierTimeout, p.step0 + b);
                                s_abort = 1;
                                ok = false;
                                break;
                            }
                        }
                        __nanosleep(32);
                    }
                }
                if (!ok)
                    break;
                __threadfence();
                if (kWords) {
                    const int w0 = (int)(((long long)c * p.nwords) / p.G);
                    const int w1 = (int)(((long long)(c + 1) * p.nwords) / p.G);
                    for (int wi = w0; wi < w1; ++wi)
                        dst[wi] = __ldcg(p.spk + (size_t)curb * p.nwords + wi);
                }
            }
            if (__any_sync(kFull, !ok))
                return;
            __syncwarp();
            if (lane == 0)
                st_release_cta(&s_gather, (int)(b + 1));
        }
        return;
    }

    if (VAR == 1 && tid >= NC) {
        if (lane != 0 || S_b == 0)
            return;
        long long q = 0;  // stages issued
        int st = 0;       // q % NST
        long long rounds = 0;  // q / NST
        bool ok = true;
        const int S_act = p.bal ? p.n / p.G + (blockIdx.x < p.n % p.G ? 1 : 0) : S_b;
        const int nbox = (S_act + p.BW - 1) / p.BW;
        // slots [0, l2_pin) stay L2-resident, the others stream through
        const unsigned long long pol_in = l2_policy(true);
        const unsigned long long pol_out = l2_policy(false);
        for (long long b = 0; b < B && ok; ++b) {
            const long long g = p.step0 + b;
            const int lim = (int)(g < L ? g : L - 1);
            if (lim < 2 + RL)
                continue;
            if (b >= 2) {
                // rows of step g are states of steps <= g-2
                unsigned long long t0 = globaltimer_ns();
                unsigned polls = 0;
                while (ld_acquire_cta(&s_done) < b - 1) {
                    if ((++polls & 63u) == 0) {
                        if (s_abort || ld_volatile_i32(p.err) != kErrNone) {
                            ok = false;
                            break;
                        }
                        if (globaltimer_ns() - t0 > p.tmo) {
                            record_err(p.err, kErrBarrierTimeout, g);
                            s_abort = 1;
                            ok = false;
                            break;
                        }
                    }
                    __nanosleep(64);
                }
                if (!ok)
                    break;
            }
            // lags k..k+cnt-1 are rows rh down to rh-cnt+1: one contiguous
            // ascending row range per stage (split at the wrap)
            SP_STAMP(true, b, B, 7);
            int rh = (int)(((g - 2 - RL) % L + L) % L);
            for (int k = 2 + RL; k <= lim && ok;) {
                int cnt = lim - k + 1;
                if (cnt > p.R)
                    cnt = p.R;
                if (cnt > rh + 1)
                    cnt = rh + 1;
                const int y0 = rh - cnt + 1;
                if (rounds > 0 &&
                    !mbar_wait(&empty[st], (unsigned)((rounds - 1) & 1), &s_abort, p.err,
                               p.tmo, g)) {
                    ok = false;
                    break;
                }
                mbar_expect_tx(&full[st], (unsigned)(nbox * p.RB * p.BW * 8));
                double *dst = s_stage + (size_t)st * STAGE;
                if (p.l2_pin > 0) {
                    // the oldest l2_pin lags stay resident: a row is read
                    // evict-first while young and turns evict-last when it
                    // reaches lag L - l2_pin (one row per step comes back
                    // from DRAM for that)
                    const unsigned long long pol = k + cnt > L - p.l2_pin ? pol_in : pol_out;
                    for (int c = 0; c < nbox; ++c)
                        tma_load_2d_hint(dst + (size_t)c * p.R * p.BW, &p.tmap, lo + c * p.BW,
                                         y0, &full[st], pol);
                } else {
                    for (int c = 0; c < nbox; ++c)
                        tma_load_2d(dst + (size_t)c * p.R * p.BW, &p.tmap, lo + c * p.BW, y0,
                                    &full[st]);
                }
                ++q;
                if (++st == p.NST) {
                    st = 0;
                    ++rounds;
                }
                k += cnt;
                rh -= cnt;
                if (rh < 0)
                    rh += L;
            }
        }
        // every issued copy must land before the CTA may exit
        const unsigned long long t0 = globaltimer_ns();
        for (long long qq = (q > p.NST ? q - p.NST : 0); qq < q; ++qq) {
            const int st = (int)(qq % p.NST);
            while (!mbar_test(&full[st], (unsigned)((qq / p.NST) & 1))) {
                if (globaltimer_ns() - t0 > p.tmo)
                    break;
            }
        }
        return;
    }

    // ------------------------------------------------------------ consumers
    const int gw = wb0 + warp;
    const bool wact = gw < wb1;
    const int i = gw * 32 + lane;
    const bool act = wact && __ldg(p.nid_of + i) >= 0;
    // ring writes: evict-first (a row is lag 34 when it is first read back)
    const unsigned long long c_pol_out = VAR == 1 ? l2_policy(false) : 0;

    double V = act ? p.V[i] : 0.0;
    double tprev = 0.0, vlast = 0.0;
    int cpos = 0;
    long long refr = 0;
    unsigned long long rng = 0;
    if (act) {
        if (NT == SP_FLIF_GL || NT == SP_FLIF_CAPUTO)
            tprev = p.tprev[i];
        if (NT == SP_FLIF_GL) {
            long long pr = (p.step0 - 1) % L;
            if (pr < 0)
                pr += L;
            vlast = p.ring[(size_t)pr * p.rs + i];
        }
    }
    // lag 2 + j of the next step: the state of micro-step step0 - 2 - j
    double hreg[RL > 0 ? RL : 1];
#pragma unroll
    for (int j = 0; j < (RL > 0 ? RL : 1); ++j)
        hreg[j] = 0.0;
    if (RL > 0 && act) {
#pragma unroll
        for (int j = 0; j < RL; ++j) {
            const long long pr = ((p.step0 - 2 - j) % L + L) % L;
            hreg[j] = p.ring[(size_t)pr * p.rs + i];
        }
    }
    if (act) {
        if (NT == SP_FLIF_CAPUTO)
            cpos = p.cap_pos[i];
        if (NT == SP_FLIF_DIFFUSIVE) {
            refr = p.refr_until[i];
            rng = p.rng[i];
        }
    }
    double ptrace = (ST == SP_SYN_PSC_HOM && act) ? p.trace[i] : 0.0;
    double Ilast = 0.0;
    if (ST == SP_SYN_FRAC && act) {
        long long pr = (p.syn_step0 - 1) % p.Ls;
        if (pr < 0)
            pr += p.Ls;
        Ilast = p.Iring[(size_t)pr * p.rs + i];
    }
    int cur = p.phase0;
    double sprev = 0.0;
    if (act)
        sprev = ((p.spk[cur * p.nwords + gw] >> lane) & 1u) ? 1.0 : 0.0;
    unsigned lastword = 0;
    int cst = 0, cph = 0;  // variant 1: stage consumed next and its phase parity
    double ext = 0.0;

    // synapse prepare for the own neuron before micro-step b (src/synapse.c:145-160)
    auto prepare = [&](long long b, int buf) {
        if (!act)
            return;
        if (ST == SP_SYN_PSC_HOM) {
            ptrace = add(mul(ptrace, p.psc_decay), mul(p.psc_omd, sprev));
            p.eff[(size_t)buf * p.rs + i] = ptrace;
        } else if (ST == SP_SYN_FRAC) {
            const long long gs = p.syn_step0 + b;
            const int Ls = p.Ls;
            const int head = (int)(gs % Ls);
            const long long lim = gs < Ls ? gs : Ls - 1;
            double hist = 0.0;
            if (lim >= 1)
                hist = add(hist, mul(__ldg(p.scoef + 1), Ilast));
            int r = head - 2;
            if (r < 0)
                r += Ls;
            for (int k = 2; k <= lim; ++k) {
                hist = add(hist, mul(__ldg(p.scoef + k), __ldcg(p.Iring + (size_t)r * p.rs + i)));
                r = (r == 0) ? Ls - 1 : r - 1;
            }
            const double rhs = dvd(add(-Ilast, sprev), p.s_tau);
            const double In = sub(mul(p.s_dta, rhs), hist);
            p.Iring[(size_t)head * p.rs + i] = In;
            Ilast = In;
            p.eff[(size_t)buf * p.rs + i] = In;
        } else if (ST == SP_SYN_FRAC_MEXP) {
            double sum = 0.0;
            for (int c = 0; c < p.Nc; ++c) {
                double tr = p.mx_tr[(size_t)c * p.rs + i];
                tr = add(mul(tr, __ldg(p.mx_decay + c)), mul(__ldg(p.mx_omd + c), sprev));
                p.mx_tr[(size_t)c * p.rs + i] = tr;
                sum = add(sum, mul(__ldg(p.mx_c + c), tr));
            }
            p.eff[(size_t)buf * p.rs + i] = sum;
        }
    };

    // arrival at the barrier that opens micro-step b
    // Grid barrier as per-CTA flags: arriving at barrier b publishes b + 1 in
    // the CTA's own flag (after its spike words); waiting, consumer thread t
    // watches the flags of CTAs t, t + NC, ... and, as soon as one is up, copies
    // that CTA's spike words into shared memory -- so the copy of the early
    // CTAs' words overlaps the wait for the late ones, and no two CTAs write
    // the same line.
    auto barrier_arrive = [&](long long b) {
        named_sync(NC);
        if (tid == 0 && p.G > 1 && !(b == p.hold_b && (int)blockIdx.x == p.hold_cta)) {
            __threadfence();
            *(volatile unsigned long long *)(p.flags + (size_t)blockIdx.x * kFlagStride) =
                (unsigned long long)(b + 1);
        }
    };
    // returns false when the launch must stop
    auto barrier_wait = [&](long long b) -> bool {
        constexpr bool kWords = ST == SP_SYN_SIMPLE || ST == SP_SYN_PSC_HET;
        const unsigned long long want = (unsigned long long)(b + 1);
        unsigned *s_spk = s_spkb + (size_t)(VAR == 1 ? (b & 1) : 0) * (spk_one / 4);
        if (VAR == 1 && p.G > 1) {
            // the gather warp has the words: wait for its announcement
            if (tid == 0) {
                if (ld_acquire_cta(&s_gather) < (int)(b + 1)) {
                    const unsigned long long t0 = globaltimer_ns();
                    unsigned polls = 0;
                    while (ld_acquire_cta(&s_gather) < (int)(b + 1)) {
                        if ((++polls & 63u) == 0) {
                            if (s_abort || ld_volatile_i32(p.err) != kErrNone)
                                break;
                            if (globaltimer_ns() - t0 > p.tmo) {
                                record_err(p.err, kErrBarrierTimeout, p.step0 + b);
                                s_abort = 1;
                                break;
                            }
                        }
                    }
                }
                if (!kWords)
                    __threadfence();  // the drive in global memory is read next
            }
        } else if (p.G > 1) {
            for (int c = tid; c < p.G; c += NC) {
                const unsigned long long *f = p.flags + (size_t)c * kFlagStride;
                if (ld_volatile_u64(f) < want) {
                    const unsigned long long t0 = globaltimer_ns();
                    unsigned long long polls = 0;
                    bool ok = true;
                    while (ld_volatile_u64(f) < want) {
                        if ((++polls & 255ull) == 0) {
                            if (s_abort || ld_volatile_i32(p.err) != kErrNone) {
                                ok = false;
                                break;
                            }
                            if (globaltimer_ns() - t0 > p.tmo || polls > kBarrierMaxPolls) {
                                record_err(p.err, kErrBarrierTimeout, p.step0 + b);
                                ok = false;
                                break;
                            }
                        }
                        __nanosleep(32);
                    }
                    if (!ok) {
                        s_abort = 1;
                        break;
                    }
                }
                __threadfence();
                if (kWords) {
                    const int w0 = (int)(((long long)c * p.nwords) / p.G);
                    const int w1 = (int)(((long long)(c + 1) * p.nwords) / p.G);
                    for (int wi = w0; wi < w1; ++wi)
                        s_spk[wi] = __ldcg(p.spk + (size_t)cur * p.nwords + wi);
                }
            }
        } else if (kWords) {
            for (int wi = tid; wi < p.nwords; wi += NC)
                s_spk[wi] = __ldcg(p.spk + (size_t)cur * p.nwords + wi);
        }
        named_sync(NC);
        // one verdict for the whole CTA (another CTA may record an error at any
        // moment; every consumer must take the same branch)
        if (tid == 0)
            s_flag = (!s_abort && ld_volatile_i32(p.err) == kErrNone) ? 1 : 0;
        named_sync(NC);
        return s_flag != 0;
    };

    // prologue: drive of micro-step 0, then arrive at barrier 0
    if (ST != SP_SYN_SIMPLE && ST != SP_SYN_PSC_HET)
        prepare(0, cur);
    barrier_arrive(0);

    for (long long b = 0; b < B; ++b) {
        const long long g = p.step0 + b;
        SP_STAMP(tid == 0, b, B, 0);
        const int s = (int)(b / p.micro);
        const int m = (int)(b % p.micro);
        if (m == 0) {
            // ext = 0 + gamma * sum_j W_in[i][j] u[j] (netlib dgemv order)
            ext = 0.0;
            if (act && p.din > 0 && p.gamma != 0.0 && p.u) {
                const double *ur = p.u + (size_t)s * p.din;
                const double *wr = p.W_in + (size_t)i * p.din;
                double t = 0.0;
                for (int j = 0; j < p.din; ++j)
                    t = add(t, mul(ldg_na(wr + j), ldg_na(ur + j)));
                ext = add(0.0, mul(p.gamma, t));
            }
        }

        // ---- FLIF_GL history sum of step g
        bool integ = false;
        double hist = 0.0;
        int head = 0;
        if (NT == SP_FLIF_GL) {
            head = (int)(g % L);
            integ = tprev > p.f;
            const int lim = (int)(g < L ? g : L - 1);
            if (act && integ && lim >= 1)
                hist = add(hist, mul(__ldg(p.coef + 1), vlast));
            if (VAR == 0) {
                if (act && integ) {
                    int r = head - 2;
                    if (r < 0)
                        r += L;
                    const double *ci = p.ring + i;
#pragma unroll 8
                    for (int k = 2; k <= lim; ++k) {
                        hist = add(hist, mul(__ldg(p.coef + k), __ldcg(ci + (size_t)r * p.rs)));
                        r = (r == 0) ? L - 1 : r - 1;
                    }
                }
            } else {
                const int boff = (tid / p.BW) * p.R * p.BW + (tid % p.BW);
                const double *cf = p.coef_smem ? s_coef : p.coef;
                if (act && integ) {
                    // lags 2 .. RL+1 from registers, in ascending order
#pragma unroll
                    for (int j = 0; j < RL; ++j)
                        if (2 + j <= lim)
                            hist = add(hist, mul(cf[2 + j], hreg[j]));
                }
                int rh = (int)(((long long)head - 2 - RL) % L + L) % L;
                for (int k = 2 + RL; k <= lim && S_b > 0;) {
                    int cnt = lim - k + 1;
                    if (cnt > p.R)
                        cnt = p.R;
                    if (cnt > rh + 1)
                        cnt = rh + 1;
                    // on a failed wait the launch aborts at the next barrier_wait;
                    // every consumer keeps the same control flow until then
                    const bool landed = mbar_wait(&full[cst], (unsigned)cph, &s_abort, p.err, p.tmo, g);
                    const double *buf = s_stage + (size_t)cst * STAGE + boff;
                    if (landed && act && integ) {
                        if ((cnt & 15) == 0) {
                            // full stages of 16, 32 or 64 rows: 16 lags at a time
                            // with their loads batched, still in ascending lag
                            // order (lag k + jr sits at row offset cnt-1-jr)
                            for (int h = 0; h < cnt; h += 16)
                                hist = stage_sum<16>(hist, cf + k + h,
                                                     buf + (size_t)(cnt - 16 - h) * p.BW, p.BW);
                        } else if ((cnt & 7) == 0) {
                            // stages of 24, 40, 48 or 56 rows: 16 at a time, then 8
                            int h = 0;
                            for (; h + 16 <= cnt; h += 16)
                                hist = stage_sum<16>(hist, cf + k + h,
                                                     buf + (size_t)(cnt - 16 - h) * p.BW, p.BW);
                            for (; h < cnt; h += 8)
                                hist = stage_sum<8>(hist, cf + k + h,
                                                    buf + (size_t)(cnt - 8 - h) * p.BW, p.BW);
                        } else {
                            for (int jr = 0; jr < cnt; ++jr)
                                hist = add(hist, mul(cf[k + jr],
                                                     buf[(size_t)(cnt - 1 - jr) * p.BW]));
                        }
                    }
                    __syncwarp();
                    if (lane == 0)
                        mbar_arrive(&empty[cst]);
                    if (++cst == p.NST) {
                        cst = 0;
                        cph ^= 1;
                    }
                    k += cnt;
                    rh -= cnt;
                    if (rh < 0)
                        rh += L;
                }
            }
        }

        // ---- barrier: spikes / eff of step g-1 are visible
        SP_STAMP(tid == 0, b, B, 1);
        if (!barrier_wait(b))
            return;
        SP_STAMP(tid == 0, b, B, 2);
        SP_STAMP(tid == 0, b, B, 3);
        const unsigned *s_spk = s_spkb + (size_t)(VAR == 1 ? (b & 1) : 0) * (spk_one / 4);

        // ---- recurrent input
        double rec = 0.0;
        if (ST == SP_SYN_SIMPLE) {
            if (wact) {
                // CSR rows are in position order; holes are empty rows
                if (p.csr_cap > 0)
                    rec = rowpass_simple_smem(s_csr_rp, s_csr_col, s_csr_w, s_spk,
                                              (gw - wb0) * 32, lane);
                else
                    rec = rowpass_simple_warp(p.row_ptr, p.col, p.w, s_spk, gw * 32, 32, lane);
            }
        } else if (wact) {
            // whole warps (holes are empty rows): every edge carries a term
            rec = rowpass_terms_warp<ST>(p, p.eff + (size_t)cur * p.rs, s_spk, gw * 32, lane);
        }

        SP_STAMP(tid == 0, b, B, 4);
        // ---- neuron update (operation order of src/neurons/<model>.c)
        bool fired = false;
        if (act) {
            const double in = add(ext, rec);
            if (NT == SP_LIF_DISCRETE) {
                V = add(add(mul(p.c, V), in), p.d);
                if (V > p.b) {
                    V = p.a;
                    fired = true;
                }
            } else if (NT == SP_LIF_BIO) {
                const double dV = dvd(add(add(-V, in), p.d), p.c);
                V = add(V, mul(dV, p.dt));
                if (V >= p.b) {
                    V = p.a;
                    fired = true;
                }
            } else if (NT == SP_FLIF_GL) {
                if (integ) {
                    const double rhs = add(add(dvd(-sub(vlast, p.c), p.d), in), p.e);
                    V = sub(mul(p.g, rhs), hist);
                    if (V >= p.a) {
                        V = p.b;
                        fired = true;
                        tprev = 0.0;
                    }
                } else {
                    V = p.b;
                }
                if (VAR == 1 && p.l2_pin > 0)
                    st_hint_f64(p.ring + (size_t)head * p.rs + i, V,
                                c_pol_out);
                else
                    p.ring[(size_t)head * p.rs + i] = V;
                if (RL > 0) {
#pragma unroll
                    for (int j = (RL > 0 ? RL : 1) - 1; j > 0; --j)
                        hreg[j] = hreg[j - 1];
                    hreg[0] = vlast;
                }
                vlast = V;
                tprev = add(tprev, p.dt);
            } else if (NT == SP_FLIF_CAPUTO) {
                if (tprev > p.f) {
                    const double dV = dvd(add(mul(-p.c, sub(V, p.d)), in), p.e);
                    const double markov = mul(p.g, dV);
                    const int D = L;
                    double *rg = p.ring + (size_t)i * D;
                    rg[cpos] = sub(V, p.b);
                    int qq = cpos;
                    cpos = (cpos + 1 == D) ? 0 : cpos + 1;
                    double mem = 0.0;
                    for (int k = 0; k < D; ++k) {
                        mem = add(mem, mul(__ldg(p.coef + k), rg[qq]));
                        qq = (qq == 0) ? D - 1 : qq - 1;
                    }
                    V = add(V, sub(markov, mem));
                    if (V >= p.a) {
                        V = p.b;
                        fired = true;
                        tprev = 0.0;
                    }
                } else {
                    V = p.b;
                }
                tprev = add(tprev, p.dt);
            } else if (NT == SP_FLIF_DIFFUSIVE) {
                const double Vp = V;
                const double rhs = add(add(-sub(Vp, p.c), in), p.d);
                V = add(Vp, mul(p.e, rhs));
                if (g >= refr && V >= p.a) {
                    V = p.b;
                    fired = true;
                    long long steps;
                    if (p.diff_sto) {
                        double W;
                        const double u0 = u01(&rng);
                        if (u0 < p.ci) {
                            W = p.h;
                        } else {
                            const double u1 = u01(&rng);
                            const double tmin = p.f, tmax = p.g, qx = p.cj;
                            if (tmax <= tmin)
                                W = tmin;
                            else if (qx <= 1e-12)
                                W = tmin + u1 * (tmax - tmin);
                            else if (fabs(qx - 1.0) < 1e-12)
                                W = tmin * pow(tmax / tmin, u1);
                            else
                                W = pow((1.0 - u1) * p.ck + u1 * p.cl, 1.0 / (1.0 - qx));
                        }
                        steps = (W <= 0.0) ? 0 : (long long)ceil(W / p.dt);
                        if (steps < 1)
                            steps = 1;
                    } else {
                        steps = p.det_refr;
                    }
                    refr = g + steps;
                }
            }
        }
        // the ring row of step g is first read by a bulk copy as lag RL + 2,
        // RL + 2 steps later: with the register lags one proxy fence per 16
        // steps orders every row before that read (kernel boundaries order
        // the rest)
        if (VAR == 1 && (RL < 32 || (g & 15) == 15))
            fence_proxy_async();

        // ---- spike word of step g
        const unsigned word = __ballot_sync(kFull, fired);
        if (wact && lane == 0)
            p.spk[(size_t)(cur ^ 1) * p.nwords + gw] = word;
        lastword = word;
        sprev = fired ? 1.0 : 0.0;
        SP_STAMP(tid == 0, b, B, 5);
        if (m == p.micro - 1) {
            if (act && p.phi)
                p.phi[(size_t)s * p.rs + i] = V;
            if (wact && lane == 0 && p.raster)
                p.raster[(size_t)s * p.nwords + gw] = lastword;
        }
        if (b + 1 < B) {
            if (ST != SP_SYN_SIMPLE && ST != SP_SYN_PSC_HET)
                prepare(b + 1, cur ^ 1);
            barrier_arrive(b + 1);
            if (VAR == 1 && tid == 0)
                st_release_cta(&s_done, (int)(b + 1));
        }
        SP_STAMP(tid == 0, b, B, 6);
        cur ^= 1;
    }

    if (act) {
        p.V[i] = V;
        if (NT == SP_FLIF_GL || NT == SP_FLIF_CAPUTO)
            p.tprev[i] = tprev;
        if (NT == SP_FLIF_CAPUTO)
            p.cap_pos[i] = cpos;
        if (NT == SP_FLIF_DIFFUSIVE) {
            p.refr_until[i] = refr;
            p.rng[i] = rng;
        }
        if (ST == SP_SYN_PSC_HOM)
            p.trace[i] = ptrace;
    }
}

}  // namespace sp
