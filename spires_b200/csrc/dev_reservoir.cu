// dev_reservoir.cu -- device state of one reservoir and the host side of the
// persistent step kernel (sp_step_kernel.cuh).
//
// Neuron layout. Device state lives in "position" space: neurons are sorted by
// CSR row length (descending) and dealt round-robin over the ceil(n/32) warps,
// rank r going to warp r % nw, lane r / nw. Every warp (and so every CTA) gets
// the same mix of long and short rows; without it a heavy-tailed graph
// (Barabasi-Albert hubs are the oldest, lowest-index nodes) puts most CSR
// edges in one warp, whose row walk then paces the whole grid every step.
// Only storage moves: each row keeps its edges in the original ascending
// column order, so every sum is formed in the reference's order, and results
// are returned in neuron order (gather kernels below).
//
// Reference for the whole loop: step_reservoir, src/reservoir.c:113-165.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <cstdio>
#include <cmath>
#include <algorithm>
#include <numeric>
#include <vector>
#include "sp_alloc.h"
#include "sp_dev.h"
#include "sp_kernels.cuh"
#include "sp_dev_internal.h"
#include "sp_step_kernel.cuh"

typedef void (*kfn_t)(sp::KP);

using namespace sp;

namespace {

template <int NT, int VAR>
kfn_t pick_syn(int st)
{
    switch (st) {
    case SP_SYN_SIMPLE: return k_run<NT, SP_SYN_SIMPLE, VAR>;
    case SP_SYN_PSC_HOM: return k_run<NT, SP_SYN_PSC_HOM, VAR>;
    case SP_SYN_PSC_HET: return k_run<NT, SP_SYN_PSC_HET, VAR>;
    case SP_SYN_FRAC: return k_run<NT, SP_SYN_FRAC, VAR>;
    case SP_SYN_FRAC_MEXP: return k_run<NT, SP_SYN_FRAC_MEXP, VAR>;
    }
    return nullptr;
}

kfn_t pick_kernel(int nt, int st, int variant)
{
    if (variant == 1)
        return nt == SP_FLIF_GL ? pick_syn<SP_FLIF_GL, 1>(st) : nullptr;
    switch (nt) {
    case SP_LIF_DISCRETE: return pick_syn<SP_LIF_DISCRETE, 0>(st);
    case SP_LIF_BIO: return pick_syn<SP_LIF_BIO, 0>(st);
    case SP_FLIF_CAPUTO: return pick_syn<SP_FLIF_CAPUTO, 0>(st);
    case SP_FLIF_GL: return pick_syn<SP_FLIF_GL, 0>(st);
    case SP_FLIF_DIFFUSIVE: return pick_syn<SP_FLIF_DIFFUSIVE, 0>(st);
    }
    return nullptr;
}

// ---------------------------------------------------------------- resets --

__global__ void k_reset_neurons(int n, int nw, int L, size_t ring_elems, int ntype,
                                double v_init, double tprev_init, double *V, double *tprev,
                                double *ring, int *cap_pos, long long *refr,
                                unsigned long long *rng, const int *nid_of,
                                unsigned long long seed)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t rs = (size_t)nw * 32;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < rs; q += stride) {
        const bool act = nid_of[q] >= 0;
        V[q] = act ? v_init : 0.0;
        if (ntype == SP_FLIF_GL || ntype == SP_FLIF_CAPUTO)
            tprev[q] = tprev_init;
        if (ntype == SP_FLIF_CAPUTO)
            cap_pos[q] = 0;
        if (ntype == SP_FLIF_DIFFUSIVE) {
            refr[q] = -1;
            // stream of neuron nid: seeded from the reservoir seed and the neuron
            // index, so it does not depend on the storage layout
            unsigned long long s =
                seed ^ (0xD1B54A32D192ED03ull * (unsigned long long)((act ? nid_of[q] : 0) + 1));
            splitmix64(&s);
            rng[q] = s;
        }
    }
    if (ring) {
        // FLIF_GL ring holds V_rest; the Caputo shift register starts at zero
        const double fill = (ntype == SP_FLIF_GL) ? v_init : 0.0;
        for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < ring_elems;
             k += stride)
            ring[k] = fill;
    }
}

// Readout y[t][o] = sum_q W_out[o][q] x[t][q] over positions: one CTA per
// (t, o), a fixed thread-strided partition and a fixed shuffle tree, so every
// path (spires_run, spires_compute_output) gets the same bits.
__global__ void __launch_bounds__(256) k_readout(const double *__restrict__ W_out,
                                                 const double *__restrict__ X, int rs, int dout,
                                                 double *__restrict__ Y)
{
    __shared__ double part[8];
    const int t = blockIdx.x, o = blockIdx.y;
    const double *x = X + (size_t)t * rs;
    const double *wr = W_out + (size_t)o * rs;
    double s = 0.0;
    for (int i = threadIdx.x; i < rs; i += 256)
        s = add(s, mul(wr[i], x[i]));
    for (int off = 16; off > 0; off >>= 1)
        s = add(s, __shfl_xor_sync(kFull, s, off));
    if ((threadIdx.x & 31) == 0)
        part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0;
        for (int k = 0; k < 8; ++k)
            r = add(r, part[k]);
        Y[(size_t)t * dout + o] = r;
    }
}

// out[t][i] = in[t][pos[i]]  (T rows; position rows have stride rs)
__global__ void k_gather_rows(const double *__restrict__ in, int rs, const int *__restrict__ pos,
                              int n, size_t T, double *__restrict__ out)
{
    const size_t total = T * (size_t)n;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
         k += (size_t)gridDim.x * blockDim.x) {
        const size_t t = k / n;
        const int i = (int)(k % n);
        out[k] = in[t * rs + pos[i]];
    }
}

// out[q] = in[nid_of[q]] (0 at holes); in has n entries, out rs
__global__ void k_scatter_vec(const double *__restrict__ in, const int *__restrict__ nid_of,
                              int rs, double *__restrict__ out)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < rs; q += gridDim.x * blockDim.x)
        out[q] = nid_of[q] >= 0 ? in[nid_of[q]] : 0.0;
}

// W_out in position space [dout][rs] <-> neuron space [dout][n]
__global__ void k_wout_to_pos(const double *__restrict__ w_nat, const int *__restrict__ nid_of,
                              int n, int rs, int dout, double *__restrict__ w_pos)
{
    const size_t total = (size_t)dout * rs;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
         k += (size_t)gridDim.x * blockDim.x) {
        const int o = (int)(k / rs), q = (int)(k % rs);
        const int i = nid_of[q];
        w_pos[k] = i >= 0 ? w_nat[(size_t)o * n + i] : 0.0;
    }
}

// spike words in neuron order (nw_out words per step) from position-space
// words (nw_in per step): bit i%32 of word i/32
__global__ void k_gather_bits(const unsigned *__restrict__ in, int nw_in,
                              const int *__restrict__ pos, int n, size_t T,
                              unsigned *__restrict__ out, int nw_out)
{
    const size_t words = (size_t)nw_out;
    const size_t total = T * words * 32;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
         k += (size_t)gridDim.x * blockDim.x) {
        const size_t t = k / (words * 32);
        const int i = (int)(k % (words * 32));
        bool b = false;
        if (i < n) {
            const int q = pos[i];
            b = (in[t * (size_t)nw_in + (q >> 5)] >> (q & 31)) & 1u;
        }
        const unsigned m = __ballot_sync(kFull, b);
        if ((threadIdx.x & 31) == 0)
            out[t * words + (i >> 5)] = m;
    }
}

__global__ void k_bits_to_double(const unsigned *words, const int *pos, int n, double *out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int q = pos[i];
        out[i] = ((words[q >> 5] >> (q & 31)) & 1u) ? 1.0 : 0.0;
    }
}

}  // namespace

// ======================================================== host C ABI ======

#define SP_CK(x)                                                                   \
    do {                                                                           \
        cudaError_t e_ = (x);                                                      \
        if (e_ != cudaSuccess) {                                                   \
            sp_dev_note_error(#x, e_);                                             \
            return (e_ == cudaErrorMemoryAllocation) ? SP_EALLOC : SP_EINTERNAL;   \
        }                                                                          \
    } while (0)

extern "C" void sp_dev_note_error(const char *what, int code)
{
    if (getenv("SPIRES_DEBUG"))
        fprintf(stderr, "spires: %s failed: %s\n", what, cudaGetErrorString((cudaError_t)code));
}

template <typename T>
static int dalloc(T **p, size_t count)
{
    *p = nullptr;
    if (count == 0)
        count = 1;
    cudaError_t e = sp_cuda_malloc((void **)p, count * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        return e == cudaErrorMemoryAllocation ? SP_EALLOC : SP_EINTERNAL;
    }
    return SP_OK;
}

template <typename T>
static int dupload(T **p, const T *h, size_t count, cudaStream_t s)
{
    int rc = dalloc(p, count);
    if (rc)
        return rc;
    if (h && count) {
        cudaError_t e = cudaMemcpyAsync(*p, h, count * sizeof(T), cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess)
            return SP_EINTERNAL;
    }
    return SP_OK;
}

static int upload_consts(sp_dev *d, const sp_host_model *m)
{
    d->nc = m->nc;
    if (m->coef && d->coef)
        SP_CK(cudaMemcpyAsync(d->coef, m->coef, (size_t)m->nc.L * sizeof(double),
                              cudaMemcpyHostToDevice, d->stream));
    return SP_OK;
}

static unsigned gather_blocks(size_t total)
{
    size_t b = (total + 255) / 256;
    return (unsigned)(b > 8192 ? 8192 : (b ? b : 1));
}

// Ring columns a CTA of this launch streams: all its positions, or -- on the
// balanced layout launched over the grid it was made for -- its active
// positions only (the first n / G (+1) of its range; the rest are holes).
static int cta_span(const sp_dev *d, const sp_launch &l)
{
    if (d->bal_G > 0 && l.ctas == d->bal_G)
        return (d->n + l.ctas - 1) / l.ctas;
    return 32 * l.warps_max;
}

// TMA box of the ring pipeline: at most 256 columns (the box limit), an even
// count (16-byte rows), NBX boxes side by side covering the CTA's span.
static void box_geometry(const sp_dev *d, const sp_launch &l, int *bw, int *nbx)
{
    const int sw = cta_span(d, l);
    *nbx = (sw + 255) / 256;
    int w = (sw + *nbx - 1) / *nbx;
    *bw = (w + 1) & ~1;
}

// SIMPLE synapse: the CTA's CSR slice (position-space row offsets, column
// positions, weights) is copied to shared memory at the start of a launch
// when its largest slice has at most kCsrSmemEdges edges, so the row pass
// after each grid barrier reads no global memory. Returns the edge capacity
// to reserve (0: rows are walked from global memory).
constexpr long long kCsrSmemEdges = 2048;

static long long csr_smem_edges(const sp_dev *d, const sp_launch &l)
{
    if (d->stype != SP_SYN_SIMPLE || !d->h_row_ptr || l.ctas < 1 || l.csr_global)
        return 0;
    const long long nw = (long long)d->nwords;
    long long mx = 0;
    for (long long b = 0; b < l.ctas; ++b) {
        const long long w0 = b * nw / l.ctas, w1 = (b + 1) * nw / l.ctas;
        const long long e = d->h_row_ptr[32 * w1] - d->h_row_ptr[32 * w0];
        if (e > mx)
            mx = e;
    }
    return mx <= kCsrSmemEdges ? (mx > 0 ? mx : 1) : 0;
}

static size_t csr_smem_bytes(long long cap, int warps_max)
{
    if (cap <= 0)
        return 0;
    const size_t rows = 32 * (size_t)warps_max + 1;
    return ((size_t)cap * 8 + 127) / 128 * 128 + ((size_t)cap * 4 + 127) / 128 * 128 +
           (rows * 4 + 127) / 128 * 128;
}

// variant 1 stages the coefficient table in shared memory up to 64 KB
static size_t coef_smem_bytes(const sp_dev *d)
{
    const size_t b = ((size_t)d->nc.L * 8 + 127) & ~(size_t)127;
    return b <= 64 * 1024 ? b : 0;
}

// dynamic shared memory of a launch shape: spike words, then (variant 1) the
// ring-row stages and their full/empty mbarriers
static size_t launch_smem(const sp_dev *d, const sp_launch &l)
{
    size_t spk = (l.variant == 1 ? 2 : 1) * (((d->nwords * 4) + 127) & ~(size_t)127) +
                 csr_smem_bytes(csr_smem_edges(d, l), l.warps_max);
    if (l.variant == 1) {
        int bw, nbx;
        box_geometry(d, l, &bw, &nbx);
        return spk + coef_smem_bytes(d) + (size_t)l.stages * nbx * l.rows * bw * sizeof(double) +
               2 * (size_t)l.stages * sizeof(unsigned long long);
    }
    return spk;
}

typedef CUresult (*encode_tiled_fn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                    const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                    const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                    CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// Tiled map of the FLIF_GL ring: dims {rs, L}, row pitch rs*8 bytes, box
// {bw, r}; out-of-range rows/columns of a box read as zero.
static int encode_ring_map(sp_dev *d, int bw, int r)
{
    if (d->tmap_bw == bw && d->tmap_r == r)
        return SP_OK;
    static encode_tiled_fn enc = nullptr;
    if (!enc) {
        void *fp = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fp, cudaEnableDefault, &q) !=
                cudaSuccess ||
            !fp)
            return SP_EINTERNAL;
        enc = (encode_tiled_fn)fp;
    }
    cuuint64_t dims[2] = {(cuuint64_t)d->rs, (cuuint64_t)d->nc.L};
    cuuint64_t strides[1] = {(cuuint64_t)d->rs * sizeof(double)};
    cuuint32_t box[2] = {(cuuint32_t)bw, (cuuint32_t)r};
    cuuint32_t estr[2] = {1, 1};
    // L2 promotion fetches whole 256-byte blocks around every row segment; on
    // the balanced layout a CTA's segment (here 136 columns, 1088 bytes) ends
    // inside a block whose rest are holes, so 256-byte promotion would pull
    // 18 % more bytes from HBM than the columns in use. 64-byte promotion
    // fetches the segment exactly; dense segments of whole blocks keep 256.
    const CUtensorMapL2promotion promo = ((size_t)bw * 8) % 256 == 0
                                             ? CU_TENSOR_MAP_L2_PROMOTION_L2_256B
                                             : CU_TENSOR_MAP_L2_PROMOTION_L2_64B;
    CUresult res = enc(&d->tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, d->ring, dims, strides, box,
                       estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, promo,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (res != CUDA_SUCCESS)
        return SP_EINTERNAL;
    d->tmap_bw = bw;
    d->tmap_r = r;
    return SP_OK;
}

static int max_smem(const sp_dev *d)
{
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, d->device);
    return v > 0 ? v : 48 * 1024;
}

// Lags kept L2-resident by the variant-1 cache hints when the launch asks for
// the automatic choice. A ring that does not fit in the L2 would miss on every
// row under plain replacement (each row is read once per step, in a cycle
// longer than the cache), so the oldest lags of every step -- 70 % of the L2
// -- are read with evict-last priority and stay resident, while younger rows
// stream through with evict-first. (N=20000, L=1024 on one B200: 490 lags,
// 24.6-24.9 us per step against 29.3 without hints; 600 lags 25.1, 700 lags
// 27.7 -- the streamed rows then evict resident ones -- and the earlier
// choice of a fixed set of ring slots at half the L2, 26.0 with a wide
// spread from launch to launch.)
static int auto_l2_pin(const sp_dev *d)
{
    const double row = (double)d->rs * sizeof(double);
    const double ring = row * d->nc.L;
    if (d->l2_bytes <= 0 || ring <= 0.75 * d->l2_bytes)
        return 0;
    const int rows = (int)(0.7 * d->l2_bytes / row);
    return rows < d->nc.L ? rows : d->nc.L;
}

extern "C" int sp_dev_l2_pin_rows(const sp_dev *d)
{
    if (d->launch.variant != 1)
        return 0;
    const int pin = d->launch.l2_pin;
    if (pin < 0)
        return auto_l2_pin(d);
    return pin < d->nc.L ? pin : d->nc.L;
}

static void default_launch(sp_dev *d)
{
    int nw = (int)d->nwords;
    sp_launch l;
    memset(&l, 0, sizeof(l));
    l.l2_pin = -1;
    if (nw <= 32) {
        l.ctas = 1;
        l.warps_max = nw;
    } else {
        int G = d->num_sms < nw ? d->num_sms : nw;
        l.ctas = G;
        l.warps_max = (nw + G - 1) / G;
        if (l.warps_max > 32)
            l.warps_max = 32;
    }
    if (d->ntype == SP_FLIF_GL && d->nc.L >= 32 && l.warps_max <= kPipeWarps) {
        // The ring stream is paced by the bytes in flight per SM (the stages
        // the consumers are not reading): long rings take the stage height of
        // 64 or 48 rows that puts the most rows in flight (ties: taller),
        // shorter rings 32-row stages. (N=20000, L=1024 on 148 SMs: 3 x 48
        // rows, 31.7 us per step, against 31.9 for 2 x 64 and 33.0 for 3 x 56,
        // whose extra bytes in flight slow the serial phase's loads more than
        // they speed the stream.)
        sp_launch best = l;
        long long best_rows = 0;
        for (int rows : {64, 48, 32}) {
            if ((rows > 32) != (d->nc.L >= 512))
                continue;
            sp_launch v = l;
            v.variant = 1;
            v.rows = rows;
            int bw, nbx;
            box_geometry(d, v, &bw, &nbx);
            const size_t stage = (size_t)v.rows * nbx * bw * sizeof(double);
            const size_t budget = (size_t)(max_smem(d) - 2 * 1024);
            const size_t spk = 2 * (((d->nwords * 4) + 127) & ~(size_t)127) +
                               coef_smem_bytes(d) +
                               csr_smem_bytes(csr_smem_edges(d, v), v.warps_max);
            long long st = budget > spk ? (long long)((budget - spk) / (stage + 16)) : 0;
            if (st > 16)
                st = 16;
            if (st >= 2 && st * rows > best_rows &&
                encode_ring_map(d, bw, v.rows < d->nc.L ? v.rows : d->nc.L) == SP_OK) {
                v.stages = (int)st;
                best = v;
                best_rows = st * rows;
            }
        }
        if (best_rows > 0) {
            l = best;
            int bw, nbx;
            box_geometry(d, l, &bw, &nbx);
            encode_ring_map(d, bw, l.rows < d->nc.L ? l.rows : d->nc.L);
        }
    }
    d->launch = l;
}


// Position layout: neurons in order of decreasing row length go, one by one,
// to the warp with the fewest CSR edges so far that still has a free lane
// (longest-processing-time assignment), lanes filled from 0. Every warp, and
// so every CTA, ends up with about the same number of edges to walk.
// pos_of[i] = position of neuron i, nid_of[q] = neuron at position q or -1.
void sp_make_layout(const sp_host_model *m, int nw, const std::vector<int> *cap,
                    std::vector<int> &pos_of, std::vector<int> &nid_of)
{
    const int n = (int)m->n;
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    auto deg = [&](int i) { return (long long)(m->row_ptr[i + 1] - m->row_ptr[i]); };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return deg(a) > deg(b); });
    pos_of.assign(n, 0);
    nid_of.assign((size_t)nw * 32, -1);
    // min-heap of (edges, warp) over warps with a free lane
    typedef std::pair<long long, int> ent;
    std::vector<ent> heap;
    heap.reserve(nw);
    for (int w = 0; w < nw; ++w)
        if (!cap || (*cap)[w] > 0)
            heap.push_back(ent(0, w));
    std::vector<int> fill(nw, 0);
    auto cmp = [](const ent &a, const ent &b) { return a > b; };
    std::make_heap(heap.begin(), heap.end(), cmp);
    for (int r = 0; r < n; ++r) {
        std::pop_heap(heap.begin(), heap.end(), cmp);
        ent e = heap.back();
        heap.pop_back();
        const int w = e.second;
        const int q = w * 32 + fill[w]++;
        pos_of[order[r]] = q;
        nid_of[q] = order[r];
        if (fill[w] < (cap ? (*cap)[w] : 32)) {
            heap.push_back(ent(e.first + deg(order[r]), w));
            std::push_heap(heap.begin(), heap.end(), cmp);
        }
    }
}

extern "C" int sp_dev_create(const sp_host_model *m, sp_dev **out)
{
    *out = nullptr;
    sp_dev *d = (sp_dev *)calloc(1, sizeof(sp_dev));
    if (!d)
        return SP_EALLOC;
    d->hold_cta = -1;
    d->hold_b = -1;
    int rc = SP_OK;
#define TRY(x)                  \
    do {                        \
        rc = (x);               \
        if (rc)                 \
            goto fail;          \
    } while (0)
    {
        cudaError_t e = cudaGetDevice(&d->device);
        if (e != cudaSuccess) {
            free(d);
            return SP_EINTERNAL;
        }
        cudaDeviceGetAttribute(&d->num_sms, cudaDevAttrMultiProcessorCount, d->device);
        cudaDeviceGetAttribute(&d->l2_bytes, cudaDevAttrL2CacheSize, d->device);
        int coop = 0;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, d->device);
        d->coop = coop;
        if (cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking) != cudaSuccess) {
            free(d);
            return SP_EINTERNAL;
        }
    }
    d->n = (int)m->n;
    d->din = (int)m->din;
    d->dout = (int)m->dout;
    d->nwords_nat = (m->n + 31) / 32;
    d->nwords = d->nwords_nat;
    // Balanced layout (FLIF_GL with at least two warps of neurons per SM):
    // every one of the SMs' CTAs gets n / SMs (+1) neurons and whole warps of
    // positions with the holes at the end of its range, so no CTA streams more
    // history than another and none streams a neighbour's columns.
    d->bal_G = 0;
    {
        const long long G = d->num_sms;
        if (m->neuron_type == SP_FLIF_GL && G > 0 && (long long)m->n >= 64 * G) {
            const long long wpc = ((long long)m->n + 32 * G - 1) / (32 * G);
            if (wpc <= kPipeWarps && G * wpc > (long long)d->nwords_nat) {
                d->bal_G = (int)G;
                d->nwords = (size_t)(G * wpc);
            }
        }
    }
    d->nw = (int)d->nwords;
    d->rs = d->nw * 32;
    d->micro = m->micro_steps;
    d->dt = m->dt;
    d->gamma = m->input_strength;
    d->ntype = m->neuron_type;
    d->stype = m->syn_type;
    d->nnz = m->nnz;
    d->nc = m->nc;
    d->sc = m->sc;
    d->seed = m->diffusive_seed;
    {
        const size_t n = m->n, rs = (size_t)d->rs, din = m->din, dout = m->dout;
        cudaStream_t s = d->stream;
        std::vector<int> pos_of, nid_of;
        std::vector<int> cap;
        if (d->bal_G > 0) {
            // CTA b: n / G (+1 for the first n % G) neurons on its first lanes
            const int G = d->bal_G, wpc = d->nw / G, n = (int)m->n;
            cap.assign(d->nw, 0);
            for (int b = 0; b < G; ++b) {
                int c = n / G + (b < n % G ? 1 : 0);
                for (int w = 0; w < wpc; ++w) {
                    const int k = c < 32 ? c : 32;
                    cap[b * wpc + w] = k;
                    c -= k;
                }
            }
        }
        sp_make_layout(m, d->nw, d->bal_G > 0 ? &cap : nullptr, pos_of, nid_of);
        // CSR in position order: row q = neuron nid_of[q], edges in their original
        // order, column index mapped to the presynaptic neuron's position
        std::vector<long long> rp(rs + 1, 0);
        std::vector<int> col(m->nnz ? m->nnz : 1);
        std::vector<double> w(m->nnz ? m->nnz : 1), ed, eo;
        if (m->syn_type == SP_SYN_PSC_HET) {
            ed.resize(m->nnz ? m->nnz : 1);
            eo.resize(m->nnz ? m->nnz : 1);
        }
        std::vector<double> win(rs * (din ? din : 1), 0.0), wout(dout * rs, 0.0);
        size_t e = 0;
        for (size_t q = 0; q < rs; ++q) {
            rp[q] = (long long)e;
            const int i = nid_of[q];
            if (i < 0)
                continue;
            for (int64_t k = m->row_ptr[i]; k < m->row_ptr[i + 1]; ++k, ++e) {
                col[e] = pos_of[m->col[k]];
                w[e] = m->w[k];
                if (m->syn_type == SP_SYN_PSC_HET) {
                    ed[e] = m->edge_decay[k];
                    eo[e] = m->edge_omd[k];
                }
            }
            for (size_t j = 0; j < din; ++j)
                win[q * din + j] = m->W_in[(size_t)i * din + j];
            for (size_t o = 0; o < dout; ++o)
                wout[o * rs + q] = m->W_out[o * n + i];
        }
        rp[rs] = (long long)e;
        TRY(dupload(&d->pos_of, pos_of.data(), n, s));
        TRY(dupload(&d->nid_of, nid_of.data(), rs, s));
        TRY(dalloc(&d->V, rs));
        TRY(dalloc(&d->tprev, rs));
        TRY(dalloc(&d->spk, 2 * d->nwords));
        TRY(dalloc(&d->bar, 4));
        d->flag_cap = 8 * (d->num_sms > 0 ? d->num_sms : 1);
        TRY(dalloc(&d->flags, (size_t)d->flag_cap * kFlagStride));
        TRY(dalloc(&d->err, 4));
        TRY(dupload(&d->row_ptr, rp.data(), rs + 1, s));
        d->h_row_ptr = (long long *)malloc((rs + 1) * sizeof(long long));
        if (!d->h_row_ptr)
            TRY(SP_EALLOC);
        memcpy(d->h_row_ptr, rp.data(), (rs + 1) * sizeof(long long));
        TRY(dupload(&d->col, col.data(), m->nnz, s));
        TRY(dupload(&d->w, w.data(), m->nnz, s));
        TRY(dupload(&d->W_in, win.data(), rs * din, s));
        TRY(dupload(&d->W_out, wout.data(), rs * dout, s));
        if (m->neuron_type == SP_FLIF_GL || m->neuron_type == SP_FLIF_CAPUTO) {
            TRY(dupload(&d->coef, m->coef, (size_t)m->nc.L, s));
            // FLIF_GL: [L][rs] time-major rows; Caputo: [rs][D] per-position registers
            d->ring_elems = rs * (size_t)m->nc.L;
            TRY(dalloc(&d->ring, d->ring_elems));
        }
        if (m->neuron_type == SP_FLIF_CAPUTO)
            TRY(dalloc(&d->cap_pos, rs));
        if (m->neuron_type == SP_FLIF_DIFFUSIVE) {
            TRY(dalloc(&d->refr_until, rs));
            TRY(dalloc(&d->rng, rs));
        }
        if (m->syn_type != SP_SYN_SIMPLE) {
            TRY(dalloc(&d->eff, 2 * rs));
            SP_CK(cudaMemsetAsync(d->eff, 0, 2 * rs * sizeof(double), s));
        }
        if (m->syn_type == SP_SYN_PSC_HOM) {
            TRY(dalloc(&d->trace, rs));
            SP_CK(cudaMemsetAsync(d->trace, 0, rs * sizeof(double), s));
        }
        if (m->syn_type == SP_SYN_PSC_HET) {
            TRY(dupload(&d->edge_decay, ed.data(), m->nnz, s));
            TRY(dupload(&d->edge_omd, eo.data(), m->nnz, s));
            TRY(dalloc(&d->edge_trace, m->nnz));
            SP_CK(cudaMemsetAsync(d->edge_trace, 0, (m->nnz ? m->nnz : 1) * sizeof(double), s));
        }
        if (m->syn_type == SP_SYN_FRAC) {
            TRY(dupload(&d->scoef, m->syn_coef, (size_t)m->sc.frac_L, s));
            TRY(dalloc(&d->Iring, rs * (size_t)m->sc.frac_L));
            SP_CK(cudaMemsetAsync(d->Iring, 0, rs * (size_t)m->sc.frac_L * sizeof(double), s));
        }
        if (m->syn_type == SP_SYN_FRAC_MEXP) {
            TRY(dupload(&d->mx_decay, m->mexp_decay, (size_t)m->sc.mexp_N, s));
            TRY(dupload(&d->mx_omd, m->mexp_omd, (size_t)m->sc.mexp_N, s));
            TRY(dupload(&d->mx_c, m->mexp_c, (size_t)m->sc.mexp_N, s));
            TRY(dalloc(&d->mx_tr, rs * (size_t)m->sc.mexp_N));
            SP_CK(cudaMemsetAsync(d->mx_tr, 0, rs * (size_t)m->sc.mexp_N * sizeof(double), s));
        }
        // staging for host-driven runs: inputs, position-space states, readouts
        size_t rows = (size_t)(128u << 20) / (rs * sizeof(double));
        if (rows < 1)
            rows = 1;
        if (rows > 8192)
            rows = 8192;
        d->chunk = rows;
        TRY(dalloc(&d->d_u, rows * (din ? din : 1)));
        TRY(dalloc(&d->d_phi, rows * rs));
        TRY(dalloc(&d->d_nat, rows * n));
        TRY(dalloc(&d->d_y, rows * (dout ? dout : 1) + 2 * (dout ? dout : 1)));
        TRY(dalloc(&d->d_spkd, n));
        TRY(dalloc(&d->d_ras, rows * d->nwords));
        TRY(dalloc(&d->d_ras_nat, rows * d->nwords_nat));
        SP_CK(cudaStreamSynchronize(s));  // host vectors above go out of scope
    }
    default_launch(d);
    TRY(sp_dev_reset_neurons(d, m));
    SP_CK(cudaMemsetAsync(d->err, 0, 4 * sizeof(int), d->stream));
    SP_CK(cudaStreamSynchronize(d->stream));
    *out = d;
    return SP_OK;
fail:
    sp_dev_destroy(d);
    return rc;
#undef TRY
}

// Give every 128-byte line of [base, base + bytes) normal L2 eviction
// priority (base 128-byte aligned, bytes a multiple of 128).
__global__ void k_l2_demote(const char *base, size_t bytes)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x * 128;
    for (size_t off = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) * 128; off < bytes;
         off += stride)
        asm volatile("applypriority.global.L2::evict_normal [%0], 128;" ::"l"(base + off)
                     : "memory");
}

extern "C" void sp_dev_destroy(sp_dev *d)
{
    if (!d)
        return;
    if (d->stream && d->ring && d->l2_hinted) {
        // ring lines the step kernel left with evict-last priority would
        // otherwise outrank every later normal line in the L2 for the rest
        // of the process: give them normal priority before the ring is freed
        const size_t bytes = d->ring_elems * sizeof(double);
        k_l2_demote<<<(unsigned)(d->num_sms > 0 ? 4 * d->num_sms : 512), 256, 0, d->stream>>>(
            (const char *)d->ring, bytes);
        cudaGetLastError();
    }
    if (d->stream)
        cudaStreamSynchronize(d->stream);
    void *bufs[] = {d->V, d->tprev, d->ring, d->cap_pos, d->refr_until, d->rng, d->spk,
                    d->row_ptr, d->col, d->w, d->coef, d->eff, d->trace, d->edge_decay,
                    d->edge_omd, d->edge_trace, d->scoef, d->Iring, d->mx_decay, d->mx_omd,
                    d->mx_c, d->mx_tr, d->W_in, d->W_out, d->d_u, d->d_phi, d->d_nat, d->d_y,
                    d->d_spkd, d->d_ras, d->d_ras_nat, d->bar, d->err, d->pos_of, d->nid_of,
                    d->flags};
    for (void *b : bufs)
        if (b)
            sp_cuda_free(b);
    if (d->stream)
        cudaStreamDestroy(d->stream);
    free(d->h_row_ptr);
    free(d);
}

extern "C" int sp_dev_reset_neurons(sp_dev *d, const sp_host_model *m)
{
    int rc = upload_consts(d, m);
    if (rc)
        return rc;
    d->step = 0;
    d->phase = 0;
    SP_CK(cudaMemsetAsync(d->spk, 0, 2 * d->nwords * sizeof(unsigned), d->stream));
    int blocks = d->num_sms * 4;
    k_reset_neurons<<<blocks, 256, 0, d->stream>>>(
        d->n, d->nw, d->nc.L, d->ring_elems, d->ntype, d->nc.v_init, d->nc.tprev_init, d->V,
        d->tprev, d->ring, d->cap_pos, d->refr_until, d->rng, d->nid_of, d->seed);
    SP_CK(cudaGetLastError());
    return SP_OK;
}

extern "C" int sp_dev_set_seed(sp_dev *d, uint64_t seed)
{
    d->seed = seed;
    return SP_OK;
}

static int check_err(sp_dev *d)
{
    int h[3] = {0, 0, 0};
    SP_CK(cudaMemcpyAsync(h, d->err, 3 * sizeof(int), cudaMemcpyDeviceToHost, d->stream));
    SP_CK(cudaStreamSynchronize(d->stream));
    if (h[0] != kErrNone) {
        const long long step =
            (long long)(((unsigned long long)(unsigned)h[2] << 32) | (unsigned)h[1]);
        d->last_err_code = h[0];
        d->last_err_step = step;
        if (getenv("SPIRES_DEBUG"))
            fprintf(stderr, "spires: device error %d at micro-step %lld\n", h[0], step);
        cudaMemsetAsync(d->err, 0, 3 * sizeof(int), d->stream);
        cudaStreamSynchronize(d->stream);
        return SP_EINTERNAL;
    }
    return SP_OK;
}

#ifdef SP_PHASE_STAMPS
// Debug builds only: the phase stamps of the last launch (see SP_STAMP).
extern "C" __attribute__((visibility("default"))) int spires_dbg_phase_stamps(void *host,
                                                                             size_t bytes)
{
    if (bytes < sizeof(g_sp_stamps))
        return -1;
    if (cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpyFromSymbol(host, g_sp_stamps, sizeof(g_sp_stamps)) != cudaSuccess)
        return -1;
    return 0;
}
#endif

extern "C" int sp_dev_set_wait_limit(sp_dev *d, double ms)
{
    if (!(ms > 0.0) || ms > 60000.0)
        return SP_EINVAL;
    d->wait_ns = (unsigned long long)(ms * 1e6);
    return SP_OK;
}

extern "C" int sp_dev_hold_arrival(sp_dev *d, int cta, long long micro_step)
{
    if (cta < 0 || micro_step < 1)
        return SP_EINVAL;
    d->hold_cta = cta;
    d->hold_b = micro_step;
    return SP_OK;
}

extern "C" int sp_dev_last_error(const sp_dev *d, int *code, long long *micro_step)
{
    if (code)
        *code = d->last_err_code;
    if (micro_step)
        *micro_step = d->last_err_step;
    return SP_OK;
}

extern "C" int sp_dev_sync(sp_dev *d)
{
    SP_CK(cudaStreamSynchronize(d->stream));
    return check_err(d);
}

extern "C" int sp_dev_launch_chunk(sp_dev *d, const double *u, size_t T, double *phi,
                                   unsigned *raster)
{
    if (T == 0)
        return SP_OK;
    sp::KP p;
    memset(&p, 0, sizeof(p));
    const sp_launch &l = d->launch;
    p.n = d->n;
    p.nwords = (int)d->nwords;
    p.din = d->din;
    p.micro = d->micro;
    p.G = l.ctas;
    p.n_macro = (int)T;
    p.phase0 = d->phase;
    p.rs = d->rs;
    p.warps = l.warps_max;
    p.R = l.variant == 1 ? l.rows : 0;
    p.NST = l.variant == 1 ? l.stages : 0;
    if (l.variant == 1) {
        box_geometry(d, l, &p.BW, &p.NBX);
        p.bal = (d->bal_G > 0 && l.ctas == d->bal_G) ? 1 : 0;
        p.RB = p.R < d->nc.L ? p.R : d->nc.L;
        p.coef_smem = coef_smem_bytes(d) > 0;
        int rc = encode_ring_map(d, p.BW, p.RB);
        if (rc)
            return rc;
        p.tmap = d->tmap;
    }
    p.step0 = d->step;
    p.syn_step0 = d->syn_step;
    p.a = d->nc.a; p.b = d->nc.b; p.c = d->nc.c; p.d = d->nc.d; p.e = d->nc.e; p.f = d->nc.f;
    p.g = d->nc.g; p.h = d->nc.h; p.ci = d->nc.i; p.cj = d->nc.j; p.ck = d->nc.k; p.cl = d->nc.l;
    p.dt = d->dt;
    p.L = d->nc.L > 0 ? d->nc.L : 1;
    p.det_refr = d->nc.det_refr_steps;
    p.diff_sto = d->nc.diff_stochastic;
    p.coef = d->coef;
    p.V = d->V; p.tprev = d->tprev; p.ring = d->ring; p.cap_pos = d->cap_pos;
    p.refr_until = d->refr_until; p.rng = d->rng; p.spk = d->spk;
    p.row_ptr = d->row_ptr; p.col = d->col; p.w = d->w; p.eff = d->eff;
    p.psc_decay = d->sc.decay; p.psc_omd = d->sc.omd; p.trace = d->trace;
    p.edge_decay = d->edge_decay; p.edge_omd = d->edge_omd; p.edge_trace = d->edge_trace;
    p.Ls = d->sc.frac_L > 0 ? d->sc.frac_L : 1;
    p.scoef = d->scoef; p.s_dta = d->sc.frac_dta; p.s_tau = d->sc.frac_tau; p.Iring = d->Iring;
    p.Nc = d->sc.mexp_N; p.mx_decay = d->mx_decay; p.mx_omd = d->mx_omd; p.mx_c = d->mx_c;
    p.mx_tr = d->mx_tr;
    p.W_in = d->W_in; p.gamma = d->gamma; p.u = u;
    p.phi = phi; p.raster = raster;
    p.bar = d->bar; p.err = d->err; p.flags = d->flags;
    p.tmo = d->wait_ns ? d->wait_ns : kBarrierTimeoutNs;
    p.l2_pin = sp_dev_l2_pin_rows(d);
    if (p.l2_pin > 0)
        d->l2_hinted = 1;
    p.hold_cta = -1;
    p.hold_b = -1;
    if (d->hold_cta >= 0 && d->hold_b >= 1 && d->hold_b < (long long)T * d->micro) {
        p.hold_cta = d->hold_cta;  // one-shot: consumed by this launch
        p.hold_b = d->hold_b;
    }
    d->hold_cta = -1;
    d->hold_b = -1;
    p.nid_of = d->nid_of;
    p.csr_cap = (int)csr_smem_edges(d, l);

    kfn_t fn = pick_kernel(d->ntype, d->stype, l.variant);
    if (!fn)
        return SP_EINVAL;
    const size_t smem = launch_smem(d, l);
    // variant 1: consumer warps, the producer warp and the gather warp
    dim3 grid(l.ctas), block(32 * (l.warps_max + (l.variant == 1 ? 2 : 0)));
    if (smem > 48 * 1024)
        SP_CK(set_max_dynamic_smem((const void *)fn));
    if (l.ctas > 1) {
        SP_CK(cudaMemsetAsync(d->flags, 0,
                              (size_t)l.ctas * kFlagStride * sizeof(unsigned long long),
                              d->stream));
        void *args[] = {&p};
        SP_CK(cudaLaunchCooperativeKernel((const void *)fn, grid, block, args, smem, d->stream));
    } else {
        fn<<<grid, block, smem, d->stream>>>(p);
        SP_CK(cudaGetLastError());
    }
    d->launches++;
    const long long micro_total = (long long)T * d->micro;
    d->step += micro_total;
    d->syn_step += micro_total;
    d->phase ^= (int)(micro_total & 1);
    return SP_OK;
}


// Stream-level launchers of the layout kernels for callers that hold raw
// device pointers (the batched path).
extern "C" int sp_launch_readout(cudaStream_t s, const double *W_pos, const double *X, int rs,
                                 size_t T, int dout, double *Y)
{
    if (T == 0 || dout == 0)
        return SP_OK;
    dim3 grid((unsigned)T, (unsigned)dout);
    k_readout<<<grid, 256, 0, s>>>(W_pos, X, rs, dout, Y);
    SP_CK(cudaGetLastError());
    return SP_OK;
}

extern "C" int sp_launch_gather_rows(cudaStream_t s, const double *pos_rows, int rs,
                                     const int *pos_of, int n, size_t T, double *nat_rows)
{
    if (T == 0 || n == 0)
        return SP_OK;
    k_gather_rows<<<gather_blocks(T * n), 256, 0, s>>>(pos_rows, rs, pos_of, n, T, nat_rows);
    SP_CK(cudaGetLastError());
    return SP_OK;
}

extern "C" int sp_launch_wout_to_pos(cudaStream_t s, const double *w_nat, const int *nid_of, int n,
                                     int rs, int dout, double *w_pos)
{
    if (dout == 0)
        return SP_OK;
    k_wout_to_pos<<<gather_blocks((size_t)dout * rs), 256, 0, s>>>(w_nat, nid_of, n, rs, dout,
                                                                    w_pos);
    SP_CK(cudaGetLastError());
    return SP_OK;
}

extern "C" int sp_dev_readout(sp_dev *d, const double *X, size_t T, double *Y)
{
    if (T == 0 || d->dout == 0)
        return SP_OK;
    dim3 grid((unsigned)T, (unsigned)d->dout);
    k_readout<<<grid, 256, 0, d->stream>>>(d->W_out, X, d->rs, d->dout, Y);
    SP_CK(cudaGetLastError());
    return SP_OK;
}

// position-space rows [T][rs] -> neuron-space rows [T][n]
extern "C" int sp_dev_gather_rows(sp_dev *d, const double *pos_rows, size_t T, double *nat_rows)
{
    if (T == 0)
        return SP_OK;
    k_gather_rows<<<gather_blocks(T * d->n), 256, 0, d->stream>>>(pos_rows, d->rs, d->pos_of,
                                                                   d->n, T, nat_rows);
    SP_CK(cudaGetLastError());
    return SP_OK;
}

extern "C" int sp_dev_run(sp_dev *d, const sp_run_args *a)
{
    const size_t T = a->T;
    const size_t n = (size_t)d->n, rs = (size_t)d->rs;
    const bool want_y = (a->h_y || a->d_y) && d->dout > 0;
    const bool want_phi = a->h_phi || a->d_phi;
    const bool phi_pos = want_phi || want_y;  // kernel writes states
    const bool want_ras = a->h_raster || a->d_raster;
    size_t chunk = T;
    if (!a->u_on_device || phi_pos || want_ras)
        chunk = d->chunk;
    if (chunk == 0)
        chunk = 1;
    for (size_t t0 = 0; t0 < T; t0 += chunk) {
        const size_t tc = (T - t0 < chunk) ? T - t0 : chunk;
        const double *u = nullptr;
        if (a->u) {
            if (a->u_on_device) {
                u = a->u + t0 * d->din;
            } else if (d->din > 0) {
                SP_CK(cudaMemcpyAsync(d->d_u, a->u + t0 * d->din, tc * d->din * sizeof(double),
                                      cudaMemcpyHostToDevice, d->stream));
                u = d->d_u;
            }
        }
        int rc = sp_dev_launch_chunk(d, u, tc, phi_pos ? d->d_phi : nullptr,
                                     want_ras ? d->d_ras : nullptr);
        if (rc)
            return rc;
        if (want_ras) {
            unsigned *dst = a->d_raster ? a->d_raster + t0 * d->nwords_nat : d->d_ras_nat;
            k_gather_bits<<<gather_blocks(tc * d->nwords_nat * 32), 256, 0, d->stream>>>(
                d->d_ras, d->nw, d->pos_of, d->n, tc, dst, (int)d->nwords_nat);
            SP_CK(cudaGetLastError());
            if (a->h_raster)
                SP_CK(cudaMemcpyAsync(a->h_raster + t0 * d->nwords_nat, dst,
                                      tc * d->nwords_nat * sizeof(unsigned),
                                      cudaMemcpyDeviceToHost, d->stream));
        }
        if (want_phi) {
            double *dst = a->d_phi ? a->d_phi + t0 * n : d->d_nat;
            rc = sp_dev_gather_rows(d, d->d_phi, tc, dst);
            if (rc)
                return rc;
            if (a->h_phi)
                SP_CK(cudaMemcpyAsync(a->h_phi + t0 * n, dst, tc * n * sizeof(double),
                                      cudaMemcpyDeviceToHost, d->stream));
        }
        if (want_y) {
            double *Y = a->d_y ? a->d_y + t0 * d->dout : d->d_y;
            rc = sp_dev_readout(d, d->d_phi, tc, Y);
            if (rc)
                return rc;
            if (a->h_y)
                SP_CK(cudaMemcpyAsync(a->h_y + t0 * d->dout, Y, tc * d->dout * sizeof(double),
                                      cudaMemcpyDeviceToHost, d->stream));
        }
        if (t0 + tc < T && (!a->u_on_device || phi_pos || want_ras))
            SP_CK(cudaStreamSynchronize(d->stream)); /* staging buffers are reused */
    }
    (void)rs;
    if (a->sync)
        return sp_dev_sync(d);
    return SP_OK;
}

extern "C" int sp_dev_read_state(sp_dev *d, double *h_V)
{
    int rc = sp_dev_gather_rows(d, d->V, 1, d->d_nat);
    if (rc)
        return rc;
    SP_CK(cudaMemcpyAsync(h_V, d->d_nat, (size_t)d->n * sizeof(double), cudaMemcpyDeviceToHost,
                          d->stream));
    return sp_dev_sync(d);
}

extern "C" int sp_dev_set_state(sp_dev *d, const double *h_V)
{
    SP_CK(cudaMemcpyAsync(d->d_nat, h_V, (size_t)d->n * sizeof(double), cudaMemcpyHostToDevice,
                          d->stream));
    k_scatter_vec<<<gather_blocks(d->rs), 256, 0, d->stream>>>(d->d_nat, d->nid_of, d->rs, d->V);
    SP_CK(cudaGetLastError());
    return sp_dev_sync(d);
}

extern "C" int sp_dev_read_spikes(sp_dev *d, double *h_spk)
{
    k_bits_to_double<<<gather_blocks(d->n), 256, 0, d->stream>>>(
        d->spk + (size_t)d->phase * d->nwords, d->pos_of, d->n, d->d_spkd);
    SP_CK(cudaGetLastError());
    SP_CK(cudaMemcpyAsync(h_spk, d->d_spkd, (size_t)d->n * sizeof(double),
                          cudaMemcpyDeviceToHost, d->stream));
    return sp_dev_sync(d);
}

extern "C" int sp_dev_compute_output(sp_dev *d, double *h_y)
{
    if (d->dout == 0)
        return SP_OK;
    int rc = sp_dev_readout(d, d->V, 1, d->d_y);
    if (rc)
        return rc;
    SP_CK(cudaMemcpyAsync(h_y, d->d_y, (size_t)d->dout * sizeof(double), cudaMemcpyDeviceToHost,
                          d->stream));
    return sp_dev_sync(d);
}

// W_out (dout x n, neuron order) in device memory -> position-space copy
extern "C" int sp_dev_w_out_from_nat(sp_dev *d, const double *dev_w_nat)
{
    k_wout_to_pos<<<gather_blocks((size_t)d->dout * d->rs), 256, 0, d->stream>>>(
        dev_w_nat, d->nid_of, d->n, d->rs, d->dout, d->W_out);
    SP_CK(cudaGetLastError());
    return SP_OK;
}

// position-space W_out -> neuron order (dout x n) in device memory
extern "C" int sp_dev_w_out_to_nat(sp_dev *d, double *dev_w_nat)
{
    k_gather_rows<<<gather_blocks((size_t)d->dout * d->n), 256, 0, d->stream>>>(
        d->W_out, d->rs, d->pos_of, d->n, (size_t)d->dout, dev_w_nat);
    SP_CK(cudaGetLastError());
    return SP_OK;
}

extern "C" int sp_dev_upload_w_out(sp_dev *d, const double *h_W_out)
{
    double *tmp = nullptr;
    SP_CK(sp_cuda_malloc(&tmp, (size_t)d->n * d->dout * sizeof(double) + 8));
    cudaMemcpyAsync(tmp, h_W_out, (size_t)d->n * d->dout * sizeof(double),
                    cudaMemcpyHostToDevice, d->stream);
    int rc = sp_dev_w_out_from_nat(d, tmp);
    cudaStreamSynchronize(d->stream);
    sp_cuda_free(tmp);
    return rc ? rc : sp_dev_sync(d);
}

extern "C" int sp_dev_download_w_out(sp_dev *d, double *h_W_out)
{
    double *tmp = nullptr;
    SP_CK(sp_cuda_malloc(&tmp, (size_t)d->n * d->dout * sizeof(double) + 8));
    int rc = sp_dev_w_out_to_nat(d, tmp);
    if (!rc)
        cudaMemcpyAsync(h_W_out, tmp, (size_t)d->n * d->dout * sizeof(double),
                        cudaMemcpyDeviceToHost, d->stream);
    cudaStreamSynchronize(d->stream);
    sp_cuda_free(tmp);
    return rc ? rc : sp_dev_sync(d);
}

extern "C" void *sp_dev_stream(sp_dev *d) { return (void *)d->stream; }

extern "C" int sp_dev_get_launch(sp_dev *d, sp_launch *l)
{
    *l = d->launch;
    return SP_OK;
}

extern "C" int sp_dev_set_launch(sp_dev *d, const sp_launch *l)
{
    if (l->ctas < 1 || l->warps_max < 1 || l->warps_max > 32 || l->l2_pin < -1)
        return SP_EINVAL;
    if ((long long)l->ctas * l->warps_max < (long long)d->nwords || l->ctas > d->flag_cap)
        return SP_EINVAL;
    if (l->variant == 1) {
        if (d->ntype != SP_FLIF_GL || l->warps_max > kPipeWarps || l->rows < 1 || l->stages < 2 ||
            l->rows > 256)
            return SP_EINVAL;
        int bw, nbx;
        box_geometry(d, *l, &bw, &nbx);
        if (encode_ring_map(d, bw, l->rows < d->nc.L ? l->rows : d->nc.L) != SP_OK)
            return SP_EINTERNAL;
    } else if (l->variant != 0) {
        return SP_EINVAL;
    }
    const size_t smem = launch_smem(d, *l);
    if (smem > (size_t)max_smem(d))
        return SP_EINVAL;
    kfn_t fn = pick_kernel(d->ntype, d->stype, l->variant);
    if (!fn)
        return SP_EINVAL;
    if (l->ctas > 1) {
        if (smem > 48 * 1024)
            SP_CK(set_max_dynamic_smem((const void *)fn));
        int per_sm = 0;
        const int threads = 32 * (l->warps_max + (l->variant == 1 ? 2 : 0));
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)fn, threads,
                                                          smem) != cudaSuccess)
            return SP_EINTERNAL;
        if (!d->coop || per_sm * d->num_sms < l->ctas)
            return SP_EINVAL;
    }
    d->launch = *l;
    return SP_OK;
}

extern "C" size_t sp_dev_nwords(const sp_dev *d) { return d->nwords_nat; }
extern "C" long long sp_dev_kernel_launches(const sp_dev *d) { return d->launches; }

// ------------------------------------------------------------- autotuner --
// Candidate launch shapes are timed from one saved state (every mutable device
// buffer and the step counters are snapshotted, and restored after each
// candidate and at the end), with zero input, `steps` macro steps each.

struct sp_snap_item {
    void *ptr;
    size_t bytes;
    void *save;
};

// Every mutable buffer of the dynamics (the step counters are kept apart):
// what the autotuner restores after each candidate and what a state
// checkpoint holds.
static void state_items(sp_dev *d, std::vector<sp_snap_item> &items)
{
    const size_t rs = (size_t)d->rs;
    items = {
        {d->V, rs * 8, nullptr},
        {d->tprev, rs * 8, nullptr},
        {d->ring, d->ring ? d->ring_elems * 8 : 0, nullptr},
        {d->cap_pos, d->cap_pos ? rs * 4 : 0, nullptr},
        {d->refr_until, d->refr_until ? rs * 8 : 0, nullptr},
        {d->rng, d->rng ? rs * 8 : 0, nullptr},
        {d->spk, 2 * d->nwords * 4, nullptr},
        {d->eff, d->eff ? 2 * rs * 8 : 0, nullptr},
        {d->trace, d->trace ? rs * 8 : 0, nullptr},
        {d->edge_trace, d->edge_trace ? d->nnz * 8 : 0, nullptr},
        {d->Iring, d->Iring ? rs * (size_t)d->sc.frac_L * 8 : 0, nullptr},
        {d->mx_tr, d->mx_tr ? rs * (size_t)d->sc.mexp_N * 8 : 0, nullptr},
    };
}

static int snapshot(sp_dev *d, std::vector<sp_snap_item> &items, bool take)
{
    if (take) {
        state_items(d, items);
        for (auto &it : items) {
            if (!it.ptr || !it.bytes)
                continue;
            if (sp_cuda_malloc(&it.save, it.bytes) != cudaSuccess)
                return SP_EALLOC;
            SP_CK(cudaMemcpyAsync(it.save, it.ptr, it.bytes, cudaMemcpyDeviceToDevice, d->stream));
        }
        return SP_OK;
    }
    for (auto &it : items)
        if (it.save)
            SP_CK(cudaMemcpyAsync(it.ptr, it.save, it.bytes, cudaMemcpyDeviceToDevice, d->stream));
    return SP_OK;
}

extern "C" int sp_dev_autotune(sp_dev *d, size_t steps)
{
    if (steps == 0)
        steps = 64;
    std::vector<sp_snap_item> items;
    const long long step0 = d->step, syn0 = d->syn_step;
    const int phase0 = d->phase;
    int rc = snapshot(d, items, true);
    std::vector<sp_launch> cand;
    const int nw = d->nw;
    std::vector<int> Gs;
    auto addG = [&](int g) {
        if (g >= 1 && g <= nw && std::find(Gs.begin(), Gs.end(), g) == Gs.end())
            Gs.push_back(g);
    };
    addG(d->num_sms < nw ? d->num_sms : nw);
    addG((nw + 1) / 2 < d->num_sms ? (nw + 1) / 2 : d->num_sms / 2);
    addG((nw + 7) / 8);
    addG((nw + 15) / 16);
    addG((nw + 31) / 32);
    for (int G : Gs) {
        sp_launch l;
        memset(&l, 0, sizeof(l));
        l.ctas = G;
        l.warps_max = (nw + G - 1) / G;
        l.l2_pin = -1;
        if (l.warps_max > 32)
            continue;
        cand.push_back(l);
        if (d->ntype == SP_FLIF_GL && d->nc.L >= 32 && l.warps_max <= kPipeWarps) {
            for (int rows : {16, 32, 64}) {
                sp_launch v = l;
                v.variant = 1;
                v.rows = rows;
                int bw, nbx;
                box_geometry(d, v, &bw, &nbx);
                const size_t stage = (size_t)rows * nbx * bw * 8;
                const size_t base = 2 * (((d->nwords * 4) + 127) & ~(size_t)127) +
                                    coef_smem_bytes(d) +
                                    csr_smem_bytes(csr_smem_edges(d, v), v.warps_max);
                const size_t budget = (size_t)(max_smem(d) - 8 * 1024);
                long long st = budget > base ? (long long)((budget - base) / (stage + 16)) : 0;
                if (st > 16)
                    st = 16;
                if (st < 2)
                    continue;
                v.stages = (int)st;
                cand.push_back(v);
                if (auto_l2_pin(d) > 0) {
                    v.l2_pin = 0;  // the same shape without cache hints
                    cand.push_back(v);
                }
            }
        }
    }
    const sp_launch keep = d->launch;
    sp_launch best = keep;
    float best_ms = 1e30f;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (!rc && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
        rc = SP_EINTERNAL;
    for (size_t c = 0; c < cand.size() && !rc; ++c) {
        if (sp_dev_set_launch(d, &cand[c]) != SP_OK)
            continue;
        cudaEventRecord(e0, d->stream);
        int r2 = sp_dev_launch_chunk(d, nullptr, steps, nullptr, nullptr);
        cudaEventRecord(e1, d->stream);
        int r3 = sp_dev_sync(d);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (!r2 && !r3 && ms < best_ms) {
            best_ms = ms;
            best = cand[c];
        }
        // back to the saved state
        snapshot(d, items, false);
        d->step = step0;
        d->syn_step = syn0;
        d->phase = phase0;
    }
    if (e0)
        cudaEventDestroy(e0);
    if (e1)
        cudaEventDestroy(e1);
    cudaStreamSynchronize(d->stream);
    for (auto &it : items)
        if (it.save)
            sp_cuda_free(it.save);
    if (rc) {
        d->launch = keep;
        return rc;
    }
    if (sp_dev_set_launch(d, &best) != SP_OK)
        d->launch = keep;
    return SP_OK;
}

// ------------------------------------------------------ state checkpoint --
// A header (the sizes the buffers depend on, then the step counters) followed
// by the state_items buffers in order. Loading checks the sizes against this
// reservoir, so a checkpoint only goes back into a reservoir of the same
// configuration.

struct sp_state_header {
    char magic[8];
    long long n, rs, ntype, stype, ring_elems, nwords, nnz, frac_L, mexp_N;
    long long step, syn_step, phase;
};

static void fill_header(const sp_dev *d, sp_state_header *h)
{
    memset(h, 0, sizeof(*h));
    memcpy(h->magic, "SPSTATE1", 8);
    h->n = d->n;
    h->rs = d->rs;
    h->ntype = d->ntype;
    h->stype = d->stype;
    h->ring_elems = (long long)d->ring_elems;
    h->nwords = (long long)d->nwords;
    h->nnz = (long long)d->nnz;
    h->frac_L = d->sc.frac_L;
    h->mexp_N = d->sc.mexp_N;
    h->step = d->step;
    h->syn_step = d->syn_step;
    h->phase = d->phase;
}

extern "C" size_t sp_dev_state_bytes(sp_dev *d)
{
    std::vector<sp_snap_item> items;
    state_items(d, items);
    size_t b = sizeof(sp_state_header);
    for (const auto &it : items)
        b += it.ptr ? it.bytes : 0;
    return b;
}

extern "C" int sp_dev_state_save(sp_dev *d, void *buf)
{
    SP_CK(cudaStreamSynchronize(d->stream)); // steps still queued belong to the state
    sp_state_header h;
    fill_header(d, &h);
    memcpy(buf, &h, sizeof(h));
    char *p = (char *)buf + sizeof(h);
    std::vector<sp_snap_item> items;
    state_items(d, items);
    for (const auto &it : items) {
        if (!it.ptr || !it.bytes)
            continue;
        SP_CK(cudaMemcpyAsync(p, it.ptr, it.bytes, cudaMemcpyDeviceToHost, d->stream));
        p += it.bytes;
    }
    SP_CK(cudaStreamSynchronize(d->stream));
    return SP_OK;
}

extern "C" int sp_dev_state_check(sp_dev *d, const void *buf)
{
    sp_state_header h, mine;
    memcpy(&h, buf, sizeof(h));
    fill_header(d, &mine);
    if (memcmp(h.magic, mine.magic, 8) != 0 || h.n != mine.n || h.rs != mine.rs ||
        h.ntype != mine.ntype || h.stype != mine.stype || h.ring_elems != mine.ring_elems ||
        h.nwords != mine.nwords || h.nnz != mine.nnz || h.frac_L != mine.frac_L ||
        h.mexp_N != mine.mexp_N || (h.phase != 0 && h.phase != 1) || h.step < 0 ||
        h.syn_step < 0)
        return SP_EINVAL;
    return SP_OK;
}

extern "C" int sp_dev_state_load(sp_dev *d, const void *buf)
{
    sp_state_header h;
    int rc = sp_dev_state_check(d, buf);
    if (rc)
        return rc;
    memcpy(&h, buf, sizeof(h));
    SP_CK(cudaStreamSynchronize(d->stream));
    const char *p = (const char *)buf + sizeof(h);
    std::vector<sp_snap_item> items;
    state_items(d, items);
    for (const auto &it : items) {
        if (!it.ptr || !it.bytes)
            continue;
        SP_CK(cudaMemcpyAsync(it.ptr, p, it.bytes, cudaMemcpyHostToDevice, d->stream));
        p += it.bytes;
    }
    SP_CK(cudaStreamSynchronize(d->stream)); // the caller's buffer may go away
    d->step = h.step;
    d->syn_step = h.syn_step;
    d->phase = (int)h.phase;
    return SP_OK;
}
