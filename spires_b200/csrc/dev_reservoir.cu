// dev_reservoir.cu -- device state of one reservoir and the persistent
// multi-step kernel that advances it.
//
// One cooperative launch runs T macro steps x (1/dt) micro-steps. Each CTA owns
// a contiguous range of whole warps of neurons; a thread owns one neuron and
// keeps its state in registers for the whole launch. Per micro-step:
//
//   1. synapse "prepare" for the thread's own neuron (needs only its own spike
//      of the previous micro-step): PSC traces, fractional current, multi-exp
//      traces -> eff[i]                               (src/synapse.c:145-160)
//   2. FLIF_GL history sum over the time-major ring (own column only)
//                                                     (src/neurons/flif_gl.c:61-72)
//   3. grid barrier: every eff[] and every spike word of the previous
//      micro-step is visible
//   4. recurrent input: ascending-column walk over the neuron's CSR row
//      (src/sparse.c:68-76); SIMPLE adds w only where the presynaptic spike
//      bit is set (w * 0.0 = +-0 leaves a sum that started at +0 unchanged)
//   5. neuron update in the reference's operation order (src/neurons/*.c)
//   6. warp ballot -> one 32-bit spike word per warp, double-buffered
//
// Reference for the whole loop: step_reservoir, src/reservoir.c:113-165.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <cstdio>
#include <cmath>
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

__global__ void k_reset_neurons(int n, int L, size_t ring_elems, int ntype, double v_init,
                                double tprev_init, double *V, double *tprev, double *ring,
                                int *cap_pos, long long *refr, unsigned long long *rng,
                                unsigned long long seed)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)n; i += stride) {
        V[i] = v_init;
        if (ntype == SP_FLIF_GL || ntype == SP_FLIF_CAPUTO)
            tprev[i] = tprev_init;
        if (ntype == SP_FLIF_CAPUTO)
            cap_pos[i] = 0;
        if (ntype == SP_FLIF_DIFFUSIVE) {
            refr[i] = -1;
            unsigned long long s = seed ^ (0xD1B54A32D192ED03ull * (i + 1));
            splitmix64(&s);
            rng[i] = s;
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

// Readout y[t][o] = sum_i W_out[o][i] x[t][i]: one CTA per (t, o), a fixed
// thread-strided partition and a fixed shuffle tree, so the result is the same
// bit pattern whichever path (spires_run, spires_compute_output) asks for it.
__global__ void __launch_bounds__(256) k_readout(const double *__restrict__ W_out,
                                                 const double *__restrict__ X, int n, int dout,
                                                 double *__restrict__ Y)
{
    __shared__ double part[8];
    const int t = blockIdx.x, o = blockIdx.y;
    const double *x = X + (size_t)t * n;
    const double *wr = W_out + (size_t)o * n;
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += 256)
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

__global__ void k_spikes_to_double(const unsigned *words, int n, double *out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = ((words[i >> 5] >> (i & 31)) & 1u) ? 1.0 : 0.0;
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
    cudaError_t e = cudaMalloc((void **)p, count * sizeof(T));
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

// dynamic shared memory of a launch shape: spike words, then (variant 1) the
// ring-row stages and their full/empty mbarriers
static size_t launch_smem(const sp_dev *d, const sp_launch &l)
{
    size_t spk = ((d->nwords * 4) + 127) & ~(size_t)127;
    if (l.variant == 1)
        return spk + (size_t)l.stages * l.rows * 32 * l.warps_max * sizeof(double) +
               2 * (size_t)l.stages * sizeof(unsigned long long);
    return spk;
}

static int max_smem(const sp_dev *d)
{
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, d->device);
    return v > 0 ? v : 48 * 1024;
}

static void default_launch(sp_dev *d)
{
    int nw = (int)d->nwords;
    sp_launch l;
    memset(&l, 0, sizeof(l));
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
    if (d->ntype == SP_FLIF_GL && d->nc.L >= 32 && l.warps_max <= 31) {
        sp_launch v = l;
        v.variant = 1;
        v.rows = 16;
        const size_t stage = (size_t)v.rows * 32 * v.warps_max * sizeof(double);
        const size_t budget = (size_t)(max_smem(d) - 8 * 1024);
        const size_t spk = ((d->nwords * 4) + 127) & ~(size_t)127;
        long long st = budget > spk ? (long long)((budget - spk) / (stage + 16)) : 0;
        if (st > 16)
            st = 16;
        if (st >= 2) {
            v.stages = (int)st;
            l = v;
        }
    }
    d->launch = l;
}

extern "C" int sp_dev_create(const sp_host_model *m, sp_dev **out)
{
    *out = nullptr;
    sp_dev *d = (sp_dev *)calloc(1, sizeof(sp_dev));
    if (!d)
        return SP_EALLOC;
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
    d->nwords = (m->n + 31) / 32;
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
        const size_t n = m->n;
        cudaStream_t s = d->stream;
        TRY(dalloc(&d->V, n));
        TRY(dalloc(&d->tprev, n));
        TRY(dalloc(&d->spk, 2 * d->nwords));
        TRY(dalloc(&d->bar, 4));
        TRY(dalloc(&d->err, 4));
        TRY(dupload(&d->row_ptr, (const long long *)m->row_ptr, n + 1, s));
        TRY(dupload(&d->col, (const int *)m->col, m->nnz, s));
        TRY(dupload(&d->w, m->w, m->nnz, s));
        TRY(dupload(&d->W_in, m->W_in, n * m->din, s));
        TRY(dupload(&d->W_out, m->W_out, n * m->dout, s));
        d->rs = (int)((n + 31) / 32 * 32);
        if (m->neuron_type == SP_FLIF_GL || m->neuron_type == SP_FLIF_CAPUTO) {
            TRY(dupload(&d->coef, m->coef, (size_t)m->nc.L, s));
            // FLIF_GL: [L][rs] time-major rows; Caputo: [n][D] per-neuron registers
            d->ring_elems = (m->neuron_type == SP_FLIF_GL) ? (size_t)d->rs * m->nc.L
                                                            : n * (size_t)m->nc.L;
            TRY(dalloc(&d->ring, d->ring_elems));
        }
        if (m->neuron_type == SP_FLIF_CAPUTO)
            TRY(dalloc(&d->cap_pos, n));
        if (m->neuron_type == SP_FLIF_DIFFUSIVE) {
            TRY(dalloc(&d->refr_until, n));
            TRY(dalloc(&d->rng, n));
        }
        if (m->syn_type != SP_SYN_SIMPLE)
            TRY(dalloc(&d->eff, 2 * n));
        if (m->syn_type == SP_SYN_PSC_HOM) {
            TRY(dalloc(&d->trace, n));
            SP_CK(cudaMemsetAsync(d->trace, 0, n * sizeof(double), s));
        }
        if (m->syn_type == SP_SYN_PSC_HET) {
            TRY(dupload(&d->edge_decay, m->edge_decay, m->nnz, s));
            TRY(dupload(&d->edge_omd, m->edge_omd, m->nnz, s));
            TRY(dalloc(&d->edge_trace, m->nnz));
            SP_CK(cudaMemsetAsync(d->edge_trace, 0, (m->nnz ? m->nnz : 1) * sizeof(double), s));
        }
        if (m->syn_type == SP_SYN_FRAC) {
            TRY(dupload(&d->scoef, m->syn_coef, (size_t)m->sc.frac_L, s));
            TRY(dalloc(&d->Iring, n * (size_t)m->sc.frac_L));
            SP_CK(cudaMemsetAsync(d->Iring, 0, n * (size_t)m->sc.frac_L * sizeof(double), s));
        }
        if (m->syn_type == SP_SYN_FRAC_MEXP) {
            TRY(dupload(&d->mx_decay, m->mexp_decay, (size_t)m->sc.mexp_N, s));
            TRY(dupload(&d->mx_omd, m->mexp_omd, (size_t)m->sc.mexp_N, s));
            TRY(dupload(&d->mx_c, m->mexp_c, (size_t)m->sc.mexp_N, s));
            TRY(dalloc(&d->mx_tr, n * (size_t)m->sc.mexp_N));
            SP_CK(cudaMemsetAsync(d->mx_tr, 0, n * (size_t)m->sc.mexp_N * sizeof(double), s));
        }
        // chunk buffers for host-driven runs: inputs, states and readouts
        size_t rows = (size_t)(128u << 20) / (n * sizeof(double));
        if (rows < 1)
            rows = 1;
        if (rows > 8192)
            rows = 8192;
        d->chunk = rows;
        TRY(dalloc(&d->d_u, rows * (m->din ? m->din : 1)));
        TRY(dalloc(&d->d_phi, rows * n));
        TRY(dalloc(&d->d_y, rows * (m->dout ? m->dout : 1)));
        TRY(dalloc(&d->d_spkd, n));
        TRY(dalloc(&d->d_ras, rows * d->nwords));
        if (cudaMallocHost((void **)&d->h_stage, rows * (m->dout ? m->dout : 1) * sizeof(double)) !=
            cudaSuccess) {
            d->h_stage = nullptr;
            rc = SP_EALLOC;
            goto fail;
        }
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

extern "C" void sp_dev_destroy(sp_dev *d)
{
    if (!d)
        return;
    if (d->stream)
        cudaStreamSynchronize(d->stream);
    void *bufs[] = {d->V, d->tprev, d->ring, d->cap_pos, d->refr_until, d->rng, d->spk,
                    d->row_ptr, d->col, d->w, d->coef, d->eff, d->trace, d->edge_decay,
                    d->edge_omd, d->edge_trace, d->scoef, d->Iring, d->mx_decay, d->mx_omd,
                    d->mx_c, d->mx_tr, d->W_in, d->W_out, d->d_u, d->d_phi, d->d_y,
                    d->d_spkd, d->d_ras, d->bar, d->err};
    for (void *b : bufs)
        if (b)
            cudaFree(b);
    if (d->h_stage)
        cudaFreeHost(d->h_stage);
    if (d->stream)
        cudaStreamDestroy(d->stream);
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
        d->n, d->nc.L, d->ring_elems, d->ntype, d->nc.v_init, d->nc.tprev_init, d->V, d->tprev,
        d->ring, d->cap_pos, d->refr_until, d->rng, d->seed);
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
    int h[2] = {0, 0};
    SP_CK(cudaMemcpyAsync(h, d->err, 2 * sizeof(int), cudaMemcpyDeviceToHost, d->stream));
    SP_CK(cudaStreamSynchronize(d->stream));
    if (h[0] != kErrNone) {
        if (getenv("SPIRES_DEBUG"))
            fprintf(stderr, "spires: device error %d at micro-step %d\n", h[0], h[1]);
        cudaMemsetAsync(d->err, 0, 2 * sizeof(int), d->stream);
        return SP_EINTERNAL;
    }
    return SP_OK;
}

extern "C" int sp_dev_sync(sp_dev *d)
{
    SP_CK(cudaStreamSynchronize(d->stream));
    return check_err(d);
}

// Launch one chunk of `T` macro steps. u, phi, raster are device pointers.
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
    p.bar = d->bar; p.err = d->err;

    kfn_t fn = pick_kernel(d->ntype, d->stype, l.variant);
    if (!fn)
        return SP_EINVAL;
    const size_t smem = launch_smem(d, l);
    dim3 grid(l.ctas), block(32 * (l.warps_max + (l.variant == 1 ? 1 : 0)));
    if (smem > 48 * 1024)
        SP_CK(cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
    if (l.ctas > 1) {
        SP_CK(cudaMemsetAsync(d->bar, 0, sizeof(unsigned), d->stream));
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

extern "C" int sp_dev_readout(sp_dev *d, const double *X, size_t T, double *Y)
{
    if (T == 0 || d->dout == 0)
        return SP_OK;
    dim3 grid((unsigned)T, (unsigned)d->dout);
    k_readout<<<grid, 256, 0, d->stream>>>(d->W_out, X, d->n, d->dout, Y);
    SP_CK(cudaGetLastError());
    return SP_OK;
}

extern "C" int sp_dev_run(sp_dev *d, const sp_run_args *a)
{
    const size_t T = a->T;
    const size_t n = (size_t)d->n;
    const bool want_y = (a->h_y || a->d_y) && d->dout > 0;
    // states are needed on the device for readouts and host copies
    const bool phi_staged = !a->d_phi && (a->h_phi || want_y);
    const bool ras_staged = !a->d_raster && a->h_raster;
    size_t chunk = T;
    if (!a->u_on_device || phi_staged || ras_staged)
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
        double *phi = a->d_phi ? a->d_phi + t0 * n : (phi_staged ? d->d_phi : nullptr);
        unsigned *ras = a->d_raster ? a->d_raster + t0 * d->nwords
                                    : (ras_staged ? d->d_ras : nullptr);
        int rc = sp_dev_launch_chunk(d, u, tc, phi, ras);
        if (rc)
            return rc;
        if (ras_staged)
            SP_CK(cudaMemcpyAsync(a->h_raster + t0 * d->nwords, ras,
                                  tc * d->nwords * sizeof(unsigned), cudaMemcpyDeviceToHost,
                                  d->stream));
        if (a->h_phi)
            SP_CK(cudaMemcpyAsync(a->h_phi + t0 * n, phi, tc * n * sizeof(double),
                                  cudaMemcpyDeviceToHost, d->stream));
        if (want_y) {
            double *Y = a->d_y ? a->d_y + t0 * d->dout : d->d_y;
            rc = sp_dev_readout(d, phi, tc, Y);
            if (rc)
                return rc;
            if (a->h_y)
                SP_CK(cudaMemcpyAsync(a->h_y + t0 * d->dout, Y, tc * d->dout * sizeof(double),
                                      cudaMemcpyDeviceToHost, d->stream));
        }
        if (t0 + tc < T && (!a->u_on_device || phi_staged || ras_staged))
            SP_CK(cudaStreamSynchronize(d->stream)); /* staging buffers are reused */
    }
    if (a->sync)
        return sp_dev_sync(d);
    return SP_OK;
}

extern "C" int sp_dev_read_state(sp_dev *d, double *h_V)
{
    SP_CK(cudaMemcpyAsync(h_V, d->V, (size_t)d->n * sizeof(double), cudaMemcpyDeviceToHost,
                          d->stream));
    return sp_dev_sync(d);
}

extern "C" int sp_dev_set_state(sp_dev *d, const double *h_V)
{
    SP_CK(cudaMemcpyAsync(d->V, h_V, (size_t)d->n * sizeof(double), cudaMemcpyHostToDevice,
                          d->stream));
    return sp_dev_sync(d);
}

extern "C" int sp_dev_read_spikes(sp_dev *d, double *h_spk)
{
    k_spikes_to_double<<<(d->n + 255) / 256, 256, 0, d->stream>>>(
        d->spk + (size_t)d->phase * d->nwords, d->n, d->d_spkd);
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

extern "C" int sp_dev_upload_w_out(sp_dev *d, const double *h_W_out)
{
    SP_CK(cudaMemcpyAsync(d->W_out, h_W_out, (size_t)d->n * d->dout * sizeof(double),
                          cudaMemcpyHostToDevice, d->stream));
    return sp_dev_sync(d);
}

extern "C" int sp_dev_download_w_out(sp_dev *d, double *h_W_out)
{
    SP_CK(cudaMemcpyAsync(h_W_out, d->W_out, (size_t)d->n * d->dout * sizeof(double),
                          cudaMemcpyDeviceToHost, d->stream));
    return sp_dev_sync(d);
}

extern "C" void *sp_dev_stream(sp_dev *d) { return (void *)d->stream; }

extern "C" int sp_dev_get_launch(sp_dev *d, sp_launch *l)
{
    *l = d->launch;
    return SP_OK;
}

extern "C" int sp_dev_set_launch(sp_dev *d, const sp_launch *l)
{
    if (l->ctas < 1 || l->warps_max < 1 || l->warps_max > 32)
        return SP_EINVAL;
    if ((long long)l->ctas * l->warps_max < (long long)d->nwords)
        return SP_EINVAL;
    if (l->variant == 1) {
        if (d->ntype != SP_FLIF_GL || l->warps_max > 31 || l->rows < 1 || l->stages < 2 ||
            l->rows > 64)
            return SP_EINVAL;
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
            SP_CK(cudaFuncSetAttribute((const void *)fn,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0;
        const int threads = 32 * (l->warps_max + (l->variant == 1 ? 1 : 0));
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)fn, threads,
                                                          smem) != cudaSuccess)
            return SP_EINTERNAL;
        if (!d->coop || per_sm * d->num_sms < l->ctas)
            return SP_EINVAL;
    }
    d->launch = *l;
    return SP_OK;
}

extern "C" size_t sp_dev_nwords(const sp_dev *d) { return d->nwords; }
extern "C" long long sp_dev_kernel_launches(const sp_dev *d) { return d->launches; }
