/*
 * api.c -- every entry point of include/spires.h (and the host side of
 * include/spires_ext.h) for the B200 library.
 *
 * Mirrors src/spires_api.c of the reference: argument checks and status codes
 * are the same (NULL handle or buffer -> SPIRES_ERR_INVALID_ARG, dt must be in
 * (0, 1] with 1/dt an integer within 1e-12, src/spires_api.c:22-75). Behind the
 * checks, construction runs on the host (construct.c) and everything that
 * advances or reads the reservoir runs on the device (dev_*.cu).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include "../../include/spires.h"
#include "../../include/spires_ext.h"
#include "sp_model.h"
#include "sp_dev.h"
#include "sp_api_internal.h"

#define SPIRES_EXPORT __attribute__((visibility("default")))

static spires_status to_status(int rc)
{
    switch (rc) {
    case SP_OK: return SPIRES_OK;
    case SP_EINVAL: return SPIRES_ERR_INVALID_ARG;
    case SP_EALLOC: return SPIRES_ERR_ALLOC;
    default: return SPIRES_ERR_INTERNAL;
    }
}

/* dt check of src/spires_api.c:28-38 */
static int dt_ok(double dt)
{
    if (dt <= 0.0 || dt > 1.0)
        return 0;
    double steps_d = 1.0 / dt;
    int steps = (int)llround(steps_d);
    if (steps < 1 || fabs(steps_d - (double)steps) > 1e-12)
        return 0;
    return 1;
}

static int model_from_config(const spires_reservoir_config *cfg, sp_host_model *m)
{
    memset(m, 0, sizeof(*m));
    if (!dt_ok(cfg->dt))
        return SP_EINVAL;
    int rc = sp_validate_config(cfg->num_neurons, cfg->num_inputs, cfg->num_outputs, cfg->dt,
                                (int)cfg->connectivity_type, (int)cfg->neuron_type,
                                cfg->neuron_params, (int)cfg->synapse_type,
                                (int)cfg->synapse_backend);
    if (rc)
        return rc;
    m->n = cfg->num_neurons;
    m->din = cfg->num_inputs;
    m->dout = cfg->num_outputs;
    m->spectral_radius = cfg->spectral_radius;
    m->ei_ratio = cfg->ei_ratio;
    m->input_strength = cfg->input_strength;
    m->connectivity = cfg->connectivity;
    m->dt = cfg->dt;
    m->conn_type = (int)cfg->connectivity_type;
    m->neuron_type = (int)cfg->neuron_type;
    m->syn_type = (int)cfg->synapse_type;
    /* the reference builds sparse storage for SPARSE and dense for any other
     * value (synapse_build_from_dense, src/synapse.c:13-38) */
    m->syn_backend = cfg->synapse_backend == SPIRES_SYNAPSE_SPARSE ? 0 : 1;
    m->neuron_params = cfg->neuron_params;
    m->synapse_params = cfg->synapse_params;
    return SP_OK;
}

/* Wrap an already built host model into a handle with device state. */
int sp_handle_from_model(sp_host_model *m, spires_reservoir **out_r)
{
    spires_reservoir *r = calloc(1, sizeof(*r));
    if (!r)
        return SP_EALLOC;
    int rc = sp_dev_create(m, &r->dev);
    if (rc) {
        free(r);
        return rc;
    }
    r->m = *m;
    memset(m, 0, sizeof(*m)); /* ownership moved */
    *out_r = r;
    return SP_OK;
}

/* ----------------------------------------------------------- lifecycle -- */

SPIRES_EXPORT spires_status spires_reservoir_create(const spires_reservoir_config *cfg,
                                                    spires_reservoir **out_r)
{
    if (!cfg || !out_r)
        return SPIRES_ERR_INVALID_ARG;
    if (!dt_ok(cfg->dt)) {
        fprintf(stderr, "dt must be in (0, 1.0] and divide 1.0 evenly\n");
        return SPIRES_ERR_INVALID_ARG;
    }
    sp_host_model m;
    int rc = model_from_config(cfg, &m);
    if (rc)
        return to_status(rc);
    rc = sp_model_build(&m);
    if (rc) {
        sp_model_free(&m);
        return rc == SP_EINVAL ? SPIRES_ERR_INVALID_ARG : SPIRES_ERR_INTERNAL;
    }
    rc = sp_handle_from_model(&m, out_r);
    if (rc) {
        sp_model_free(&m);
        return to_status(rc);
    }
    return SPIRES_OK;
}

SPIRES_EXPORT void spires_reservoir_destroy(spires_reservoir *r)
{
    if (!r)
        return;
    sp_dev_destroy(r->dev);
    sp_model_free(&r->m);
    free(r);
}

SPIRES_EXPORT spires_status spires_reservoir_reset(spires_reservoir *r)
{
    if (!r || !r->dev)
        return SPIRES_ERR_INVALID_ARG;
    /* neuron parameters are re-read through the caller's pointer, as
     * reset_reservoir re-runs init_neuron (src/reservoir.c:770-780) */
    int rc = sp_model_derive_neuron(&r->m);
    if (rc)
        return to_status(rc);
    return to_status(sp_dev_reset_neurons(r->dev, &r->m));
}

/* ------------------------------------------------------------ stepping -- */

SPIRES_EXPORT spires_status spires_step(spires_reservoir *r, const double *u_t)
{
    if (!r || !r->dev)
        return SPIRES_ERR_INVALID_ARG;
    sp_run_args a;
    memset(&a, 0, sizeof(a));
    a.u = u_t; /* NULL = zero input vector */
    a.T = 1;
    return to_status(sp_dev_run(r->dev, &a));
}

SPIRES_EXPORT double *spires_run(spires_reservoir *r, const double *input_series,
                                 size_t series_length)
{
    if (!r || !r->dev || !input_series)
        return NULL;
    size_t count = r->m.dout * series_length;
    double *out = malloc((count ? count : 1) * sizeof(double));
    if (!out)
        return NULL;
    sp_run_args a;
    memset(&a, 0, sizeof(a));
    a.u = input_series;
    a.T = series_length;
    a.h_y = r->m.dout ? out : NULL;
    a.sync = 1;
    if (sp_dev_run(r->dev, &a) != SP_OK) {
        free(out);
        return NULL;
    }
    return out;
}

/* ------------------------------------------------------------ training -- */

SPIRES_EXPORT spires_status spires_train_online(spires_reservoir *r, const double *target_vec,
                                                double lr)
{
    if (!r || !r->dev || !target_vec)
        return SPIRES_ERR_INVALID_ARG;
    return to_status(sp_dev_train_online(r->dev, target_vec, lr, r->m.W_out));
}

SPIRES_EXPORT spires_status spires_train_ridge(spires_reservoir *r, const double *input_series,
                                               const double *target_series,
                                               size_t series_length, double lambda)
{
    if (!r || !r->dev || !input_series || !target_series)
        return SPIRES_ERR_INVALID_ARG;
    sp_ridge_opts o;
    memset(&o, 0, sizeof(o));
    o.gram_mode = sp_default_gram_mode();
    o.max_refine = 30;
    o.refine_tol = 1e-13;
    sp_ridge_report rep;
    int rc = sp_model_derive_neuron(&r->m); /* train_ridge starts with a reset */
    if (rc)
        return to_status(rc);
    rc = sp_dev_train_ridge(r->dev, &r->m, input_series, target_series, series_length, lambda,
                            &o, &rep, r->m.W_out);
    return to_status(rc);
}

SPIRES_EXPORT spires_status spires_train_rls(spires_reservoir *r, const double *input_series,
                                             const double *target_series, size_t series_length,
                                             double delta, double lambda)
{
    if (!r || !r->dev || !input_series || !target_series)
        return SPIRES_ERR_INVALID_ARG;
    int rc = sp_model_derive_neuron(&r->m);
    if (rc)
        return to_status(rc);
    return to_status(sp_dev_train_rls(r->dev, &r->m, input_series, target_series, series_length,
                                      delta, lambda, r->m.W_out));
}

/* --------------------------------------------------------------- state -- */

SPIRES_EXPORT double *spires_copy_reservoir_state(spires_reservoir *r)
{
    if (!r || !r->dev)
        return NULL;
    double *s = malloc(r->m.n * sizeof(double));
    if (!s)
        return NULL;
    if (sp_dev_read_state(r->dev, s) != SP_OK) {
        free(s);
        return NULL;
    }
    return s;
}

SPIRES_EXPORT spires_status spires_read_reservoir_state(spires_reservoir *r, double *buffer)
{
    if (!r || !r->dev || !buffer) {
        fprintf(stderr, "Error reading reservoir state, buffer not initialized!\n");
        return SPIRES_ERR_INVALID_ARG;
    }
    return to_status(sp_dev_read_state(r->dev, buffer));
}

SPIRES_EXPORT spires_status spires_read_spike_state(spires_reservoir *r, double *buffer)
{
    if (!r || !r->dev || !buffer)
        return SPIRES_ERR_INVALID_ARG;
    return to_status(sp_dev_read_spikes(r->dev, buffer));
}

static void dense_from_csr(const sp_host_model *m, double *buf)
{
    size_t n = m->n;
    memset(buf, 0, n * n * sizeof(double));
    for (size_t i = 0; i < n; i++)
        for (int64_t k = m->row_ptr[i]; k < m->row_ptr[i + 1]; k++)
            buf[i * n + (size_t)m->col[k]] = m->w[k];
}

SPIRES_EXPORT double *spires_copy_weights(const spires_reservoir *r)
{
    if (!r || !r->m.n)
        return NULL;
    double *buf = malloc(r->m.n * r->m.n * sizeof(double));
    if (!buf)
        return NULL;
    dense_from_csr(&r->m, buf);
    return buf;
}

SPIRES_EXPORT spires_status spires_read_weights(const spires_reservoir *r, double *buffer)
{
    if (!r || !buffer)
        return SPIRES_ERR_INVALID_ARG;
    if (r->m.n)
        dense_from_csr(&r->m, buffer);
    return SPIRES_OK;
}

SPIRES_EXPORT double *spires_copy_readout(const spires_reservoir *r)
{
    if (!r)
        return NULL;
    size_t cnt = r->m.dout * r->m.n;
    double *buf = malloc((cnt ? cnt : 1) * sizeof(double));
    if (!buf)
        return NULL;
    memcpy(buf, r->m.W_out, cnt * sizeof(double));
    return buf;
}

SPIRES_EXPORT spires_status spires_read_readout(const spires_reservoir *r, double *buffer)
{
    if (!r || !buffer)
        return SPIRES_ERR_INVALID_ARG;
    memcpy(buffer, r->m.W_out, r->m.dout * r->m.n * sizeof(double));
    return SPIRES_OK;
}

SPIRES_EXPORT spires_status spires_compute_output(spires_reservoir *r, double *out)
{
    if (!r || !r->dev || !out)
        return SPIRES_ERR_INVALID_ARG;
    return to_status(sp_dev_compute_output(r->dev, out));
}

SPIRES_EXPORT size_t spires_num_neurons(const spires_reservoir *r) { return r ? r->m.n : 0; }
SPIRES_EXPORT size_t spires_num_inputs(const spires_reservoir *r) { return r ? r->m.din : 0; }
SPIRES_EXPORT size_t spires_num_outputs(const spires_reservoir *r) { return r ? r->m.dout : 0; }

/* -------------------------------------------------------- extensions -- */

struct spires_ext_model {
    sp_host_model m;
};

SPIRES_EXPORT spires_status spires_ext_model_build(const spires_reservoir_config *cfg,
                                                   spires_ext_model **out)
{
    if (!cfg || !out)
        return SPIRES_ERR_INVALID_ARG;
    spires_ext_model *h = calloc(1, sizeof(*h));
    if (!h)
        return SPIRES_ERR_ALLOC;
    int rc = model_from_config(cfg, &h->m);
    h->m.host_only = 1; /* inspection builds never touch a GPU */
    if (!rc)
        rc = sp_model_build(&h->m);
    if (rc) {
        sp_model_free(&h->m);
        free(h);
        return to_status(rc);
    }
    *out = h;
    return SPIRES_OK;
}

SPIRES_EXPORT void spires_ext_model_free(spires_ext_model *h)
{
    if (!h)
        return;
    sp_model_free(&h->m);
    free(h);
}

static void fill_info(const sp_host_model *m, spires_ext_model_info *info)
{
    memset(info, 0, sizeof(*info));
    info->num_neurons = m->n;
    info->num_inputs = m->din;
    info->num_outputs = m->dout;
    info->nnz = m->nnz;
    info->ring_len = m->nc.L;
    info->micro_steps = m->micro_steps;
    info->syn_ring_len = m->sc.frac_L;
    info->syn_components = m->sc.mexp_N;
    info->spectral_radius_before_rescale = m->spectral_radius_before;
    info->topology_ms = m->topology_ms;
    info->spectral_ms = m->spectral_ms;
}

SPIRES_EXPORT spires_status spires_ext_model_info_get(const spires_ext_model *h,
                                                      spires_ext_model_info *info)
{
    if (!h || !info)
        return SPIRES_ERR_INVALID_ARG;
    fill_info(&h->m, info);
    return SPIRES_OK;
}

SPIRES_EXPORT spires_status spires_ext_model_csr(const spires_ext_model *h, int64_t *row_ptr,
                                                 int32_t *col, double *val)
{
    if (!h)
        return SPIRES_ERR_INVALID_ARG;
    const sp_host_model *m = &h->m;
    if (row_ptr)
        memcpy(row_ptr, m->row_ptr, (m->n + 1) * sizeof(int64_t));
    if (col)
        memcpy(col, m->col, m->nnz * sizeof(int32_t));
    if (val)
        memcpy(val, m->w, m->nnz * sizeof(double));
    return SPIRES_OK;
}

SPIRES_EXPORT spires_status spires_ext_model_w_in(const spires_ext_model *h, double *w_in)
{
    if (!h || !w_in)
        return SPIRES_ERR_INVALID_ARG;
    memcpy(w_in, h->m.W_in, h->m.n * h->m.din * sizeof(double));
    return SPIRES_OK;
}

SPIRES_EXPORT spires_status spires_ext_model_w_out(const spires_ext_model *h, double *w_out)
{
    if (!h || !w_out)
        return SPIRES_ERR_INVALID_ARG;
    memcpy(w_out, h->m.W_out, h->m.n * h->m.dout * sizeof(double));
    return SPIRES_OK;
}

SPIRES_EXPORT spires_status spires_ext_model_edge_tau(const spires_ext_model *h, double *tau)
{
    if (!h || !tau || !h->m.edge_tau)
        return SPIRES_ERR_INVALID_ARG;
    memcpy(tau, h->m.edge_tau, h->m.nnz * sizeof(double));
    return SPIRES_OK;
}

SPIRES_EXPORT spires_status spires_ext_model_coef(const spires_ext_model *h, double *coef)
{
    if (!h || !coef || !h->m.coef)
        return SPIRES_ERR_INVALID_ARG;
    memcpy(coef, h->m.coef, (size_t)h->m.nc.L * sizeof(double));
    return SPIRES_OK;
}

SPIRES_EXPORT spires_status spires_ext_run_record(spires_reservoir *r, const double *u, size_t T,
                                                  double *phi, uint32_t *raster, double *y)
{
    if (!r || !r->dev)
        return SPIRES_ERR_INVALID_ARG;
    sp_run_args a;
    memset(&a, 0, sizeof(a));
    a.u = u;
    a.T = T;
    a.h_phi = phi;
    a.h_raster = raster;
    a.h_y = (y && r->m.dout) ? y : NULL;
    a.sync = 1;
    return to_status(sp_dev_run(r->dev, &a));
}

SPIRES_EXPORT spires_status spires_ext_run_device(spires_reservoir *r, const double *d_u,
                                                  size_t T, double *d_phi, uint32_t *d_raster,
                                                  double *d_y)
{
    if (!r || !r->dev)
        return SPIRES_ERR_INVALID_ARG;
    sp_run_args a;
    memset(&a, 0, sizeof(a));
    a.u = d_u;
    a.u_on_device = 1;
    a.T = T;
    a.d_phi = d_phi;
    a.d_raster = d_raster;
    a.d_y = (d_y && r->m.dout) ? d_y : NULL;
    return to_status(sp_dev_run(r->dev, &a));
}

SPIRES_EXPORT spires_status spires_ext_sync(spires_reservoir *r)
{
    if (!r || !r->dev)
        return SPIRES_ERR_INVALID_ARG;
    return to_status(sp_dev_sync(r->dev));
}

SPIRES_EXPORT void *spires_ext_stream(spires_reservoir *r)
{
    return (r && r->dev) ? sp_dev_stream(r->dev) : NULL;
}

SPIRES_EXPORT size_t spires_ext_spike_words(const spires_reservoir *r)
{
    return r ? (r->m.n + 31) / 32 : 0;
}

SPIRES_EXPORT long long spires_ext_kernel_launches(const spires_reservoir *r)
{
    return (r && r->dev) ? sp_dev_kernel_launches(r->dev) : 0;
}

SPIRES_EXPORT spires_status spires_ext_read_w_in(const spires_reservoir *r, double *w_in)
{
    if (!r || !w_in)
        return SPIRES_ERR_INVALID_ARG;
    memcpy(w_in, r->m.W_in, r->m.n * r->m.din * sizeof(double));
    return SPIRES_OK;
}

SPIRES_EXPORT spires_status spires_ext_get_launch(const spires_reservoir *r,
                                                  spires_ext_launch *l)
{
    if (!r || !r->dev || !l)
        return SPIRES_ERR_INVALID_ARG;
    sp_launch s;
    sp_dev_get_launch(r->dev, &s);
    l->ctas = s.ctas;
    l->warps_max = s.warps_max;
    l->variant = s.variant;
    l->stages = s.stages;
    l->rows = s.rows;
    l->csr_global = s.csr_global;
    l->l2_pin = s.l2_pin;
    return SPIRES_OK;
}

SPIRES_EXPORT int spires_ext_l2_pin_rows(const spires_reservoir *r)
{
    if (!r || !r->dev)
        return 0;
    return sp_dev_l2_pin_rows(r->dev);
}

SPIRES_EXPORT spires_status spires_ext_set_launch(spires_reservoir *r,
                                                  const spires_ext_launch *l)
{
    if (!r || !r->dev || !l)
        return SPIRES_ERR_INVALID_ARG;
    sp_launch s = {l->ctas,   l->warps_max,          l->variant, l->stages,
                   l->rows,   l->csr_global != 0,    l->l2_pin};
    return to_status(sp_dev_set_launch(r->dev, &s));
}

SPIRES_EXPORT spires_status spires_ext_autotune(spires_reservoir *r, size_t steps)
{
    if (!r || !r->dev)
        return SPIRES_ERR_INVALID_ARG;
    return to_status(sp_dev_autotune(r->dev, steps));
}

SPIRES_EXPORT spires_status spires_ext_set_seed(spires_reservoir *r, uint64_t seed)
{
    if (!r || !r->dev)
        return SPIRES_ERR_INVALID_ARG;
    return to_status(sp_dev_set_seed(r->dev, seed));
}

/* bounded waits and failure-path test hooks */
long long sp_alloc_live(void);
void      sp_alloc_fail_after(long long count);

SPIRES_EXPORT spires_status spires_ext_set_wait_limit(spires_reservoir *r, double ms)
{
    if (!r || !r->dev)
        return SPIRES_ERR_INVALID_ARG;
    return to_status(sp_dev_set_wait_limit(r->dev, ms));
}

SPIRES_EXPORT spires_status spires_ext_test_withhold_arrival(spires_reservoir *r, int cta,
                                                             long long micro_step)
{
    if (!r || !r->dev)
        return SPIRES_ERR_INVALID_ARG;
    return to_status(sp_dev_hold_arrival(r->dev, cta, micro_step));
}

SPIRES_EXPORT spires_status spires_ext_last_device_error(const spires_reservoir *r, int *code,
                                                         long long *micro_step)
{
    if (!r || !r->dev)
        return SPIRES_ERR_INVALID_ARG;
    return to_status(sp_dev_last_error(r->dev, code, micro_step));
}

SPIRES_EXPORT void spires_ext_test_fail_device_alloc(long long after)
{
    sp_alloc_fail_after(after);
}

SPIRES_EXPORT long long spires_ext_test_live_device_allocs(void)
{
    return sp_alloc_live();
}

/* state checkpoint: a model header (sizes, micro-steps and a hash of
 * everything the dynamics read), the device state (sp_dev_state_*), then
 * W_out [dout x n]. */
typedef struct {
    char     magic[8];
    uint64_t total_bytes;
    uint64_t n, din, dout;
    int64_t  micro, neuron_type, syn_type, syn_backend;
    uint64_t model_hash;
} sp_ckpt_header;

/* FNV-1a (64-bit) over a byte range */
static uint64_t fnv1a(uint64_t h, const void *p, size_t bytes)
{
    const unsigned char *c = (const unsigned char *)p;
    for (size_t k = 0; k < bytes; ++k) {
        h ^= c[k];
        h *= 1099511628211ull;
    }
    return h;
}

#define HASH_FIELD(h, x) (h) = fnv1a((h), &(x), sizeof(x))

/* Identity of the dynamics a checkpoint belongs to: dt, the derived neuron and
 * synapse constants (which follow the current parameter arrays), the recurrent
 * CSR, W_in and the history coefficients. Two reservoirs with the same hash
 * step the same state to the same next state. */
static uint64_t model_hash(const sp_host_model *m)
{
    uint64_t h = 14695981039346656037ull;
    const sp_neuron_consts *nc = &m->nc;
    const sp_synapse_consts *sc = &m->sc;
    HASH_FIELD(h, m->dt);
    HASH_FIELD(h, m->input_strength);
    h = fnv1a(h, &nc->a, 12 * sizeof(double));
    HASH_FIELD(h, nc->v_init);
    HASH_FIELD(h, nc->tprev_init);
    HASH_FIELD(h, nc->L);
    HASH_FIELD(h, nc->det_refr_steps);
    HASH_FIELD(h, nc->diff_stochastic);
    HASH_FIELD(h, sc->decay);
    HASH_FIELD(h, sc->omd);
    HASH_FIELD(h, sc->frac_dta);
    HASH_FIELD(h, sc->frac_tau);
    HASH_FIELD(h, sc->frac_L);
    HASH_FIELD(h, sc->mexp_N);
    HASH_FIELD(h, m->diffusive_seed);
    if (m->row_ptr)
        h = fnv1a(h, m->row_ptr, (m->n + 1) * sizeof(int64_t));
    if (m->col)
        h = fnv1a(h, m->col, m->nnz * sizeof(int32_t));
    if (m->w)
        h = fnv1a(h, m->w, m->nnz * sizeof(double));
    if (m->W_in)
        h = fnv1a(h, m->W_in, m->n * m->din * sizeof(double));
    if (m->coef && nc->L > 0)
        h = fnv1a(h, m->coef, (size_t)nc->L * sizeof(double));
    if (m->edge_decay)
        h = fnv1a(h, m->edge_decay, m->nnz * sizeof(double));
    if (m->syn_coef && sc->frac_L > 0)
        h = fnv1a(h, m->syn_coef, (size_t)sc->frac_L * sizeof(double));
    if (m->mexp_decay && sc->mexp_N > 0) {
        h = fnv1a(h, m->mexp_decay, (size_t)sc->mexp_N * sizeof(double));
        h = fnv1a(h, m->mexp_c, (size_t)sc->mexp_N * sizeof(double));
    }
    return h;
}

static void ckpt_header(const spires_reservoir *r, size_t total, sp_ckpt_header *h)
{
    memset(h, 0, sizeof(*h));
    memcpy(h->magic, "SPCKPT02", 8);
    h->total_bytes = total;
    h->n = r->m.n;
    h->din = r->m.din;
    h->dout = r->m.dout;
    h->micro = r->m.micro_steps;
    h->neuron_type = r->m.neuron_type;
    h->syn_type = r->m.syn_type;
    h->syn_backend = r->m.syn_backend;
    h->model_hash = model_hash(&r->m);
}

SPIRES_EXPORT size_t spires_ext_state_bytes(spires_reservoir *r)
{
    if (!r || !r->dev)
        return 0;
    return sizeof(sp_ckpt_header) + sp_dev_state_bytes(r->dev) +
           r->m.dout * r->m.n * sizeof(double);
}

SPIRES_EXPORT spires_status spires_ext_state_save(spires_reservoir *r, void *buf,
                                                  size_t buf_bytes)
{
    if (!r || !r->dev || !buf)
        return SPIRES_ERR_INVALID_ARG;
    const size_t total = spires_ext_state_bytes(r);
    if (buf_bytes < total)
        return SPIRES_ERR_INVALID_ARG;
    sp_ckpt_header h;
    ckpt_header(r, total, &h);
    memcpy(buf, &h, sizeof(h));
    char *p = (char *)buf + sizeof(h);
    int rc = sp_dev_state_save(r->dev, p);
    if (rc)
        return to_status(rc);
    memcpy(p + sp_dev_state_bytes(r->dev), r->m.W_out, r->m.dout * r->m.n * sizeof(double));
    return SPIRES_OK;
}

SPIRES_EXPORT spires_status spires_ext_state_load(spires_reservoir *r, const void *buf,
                                                  size_t buf_bytes)
{
    if (!r || !r->dev || !buf)
        return SPIRES_ERR_INVALID_ARG;
    /* every check comes before anything of the reservoir is touched */
    const size_t total = spires_ext_state_bytes(r);
    if (buf_bytes != total || buf_bytes < sizeof(sp_ckpt_header))
        return SPIRES_ERR_INVALID_ARG;
    sp_ckpt_header h, mine;
    memcpy(&h, buf, sizeof(h));
    ckpt_header(r, total, &mine);
    if (memcmp(&h, &mine, sizeof(h)) != 0)
        return SPIRES_ERR_INVALID_ARG;
    const char *p = (const char *)buf + sizeof(h);
    int rc = sp_dev_state_check(r->dev, p);
    if (rc)
        return to_status(rc);
    rc = sp_dev_state_load(r->dev, p);
    if (rc)
        return to_status(rc);
    const size_t wb = r->m.dout * r->m.n * sizeof(double);
    if (wb) {
        memcpy(r->m.W_out, p + sp_dev_state_bytes(r->dev), wb);
        rc = sp_dev_upload_w_out(r->dev, r->m.W_out);
    }
    return to_status(rc);
}

SPIRES_EXPORT spires_status spires_ext_train_ridge(spires_reservoir *r,
                                                   const double *input_series,
                                                   const double *target_series,
                                                   size_t series_length, double lambda,
                                                   const spires_ext_ridge_opts *opts,
                                                   spires_ext_ridge_report *report)
{
    if (!r || !r->dev || !input_series || !target_series)
        return SPIRES_ERR_INVALID_ARG;
    sp_ridge_opts o;
    memset(&o, 0, sizeof(o));
    o.gram_mode = sp_default_gram_mode();
    o.max_refine = 30;
    o.refine_tol = 1e-13;
    if (opts) {
        o.gram_mode = opts->gram_mode;
        o.max_refine = opts->max_refine;
        o.refine_tol = opts->refine_tol;
        o.washout = opts->washout;
        o.gram_slices = opts->gram_slices;
    }
    if (o.washout >= series_length)
        return SPIRES_ERR_INVALID_ARG;
    sp_ridge_report rep;
    memset(&rep, 0, sizeof(rep));
    int rc = sp_model_derive_neuron(&r->m);
    if (rc)
        return to_status(rc);
    rc = sp_dev_train_ridge(r->dev, &r->m, input_series, target_series, series_length, lambda,
                            &o, &rep, r->m.W_out);
    if (report) {
        report->gram_mode_used = rep.gram_mode_used;
        report->refine_iters = rep.refine_iters;
        report->rel_residual = rep.rel_residual;
        report->collect_ms = rep.collect_ms;
        report->gram_ms = rep.gram_ms;
        report->factor_ms = rep.factor_ms;
        report->refine_ms = rep.refine_ms;
        report->factor_failed = rep.factor_failed;
        report->lu_fallback = rep.lu_fallback;
        report->dual = rep.dual;
        report->solve_ms = rep.solve_ms;
    }
    return to_status(rc);
}

/* ---- batched multi-reservoir path ---------------------------------------- */
struct spires_ext_batch {
    sp_batch *b;
    size_t count;
    double construct_ms; /* host construction of every instance */
    double setup_ms;     /* layouts, recurrent-input formats, device uploads */
};

static double now_ms(void)
{
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return 1e3 * (double)t.tv_sec + 1e-6 * (double)t.tv_nsec;
}

/* Rough host time of one build, only to order the builds of a batch: per
 * pair drawn (Erdos-Renyi), per ring edge (small-world), per roulette pick
 * (scale-free), plus the host power iteration of graphs small enough to keep
 * it on the host (1000 sweeps of their edges). */
typedef struct {
    double cost;
    size_t index;
} build_job;

static double build_cost(const spires_reservoir_config *c)
{
    const double n = (double)c->num_neurons;
    const double conn = c->connectivity > 0.0 ? (c->connectivity < 1.0 ? c->connectivity : 1.0)
                                              : 0.0;
    const double deg = conn * (n > 1.0 ? n - 1.0 : 0.0) + 1.0, edges = n * deg;
    double t;
    switch ((int)c->connectivity_type) {
    case SP_CONN_RANDOM: t = 6e-9 * n * n + 2e-8 * edges; break;
    case SP_CONN_SMALL_WORLD: t = 4e-8 * edges; break;
    default: t = 1.2e-7 * edges; break;
    }
    if (edges < 32768.0)
        t += 6e-7 * edges;
    return t;
}

static int cmp_build_job(const void *a, const void *b)
{
    const build_job *x = a, *y = b;
    if (x->cost != y->cost)
        return x->cost > y->cost ? -1 : 1;
    return (x->index > y->index) - (x->index < y->index);
}

SPIRES_EXPORT spires_status spires_ext_batch_create(const spires_reservoir_config *cfgs,
                                                    const unsigned *seeds, size_t count,
                                                    spires_ext_batch **out)
{
    if (!cfgs || !out || count == 0)
        return SPIRES_ERR_INVALID_ARG;
    *out = NULL;
    sp_host_model *ms = calloc(count, sizeof(*ms));
    spires_ext_batch *h = calloc(1, sizeof(*h));
    if (!ms || !h) {
        free(ms);
        free(h);
        return SPIRES_ERR_ALLOC;
    }
    int rc = SP_OK;
    const double t0 = now_ms();
    if (seeds) {
        /* Independent private generators: instances build on all host threads,
         * the costliest first so that no large build starts last (the order
         * changes no instance: each draws from its own generator). */
        const int dev = sp_dev_current_device();
        int *rcs = calloc(count, sizeof(int));
        build_job *jobs = malloc(count * sizeof(build_job));
        if (!rcs || !jobs) {
            free(rcs);
            free(jobs);
            free(ms);
            free(h);
            return SPIRES_ERR_ALLOC;
        }
        for (size_t k = 0; k < count; ++k) {
            jobs[k].cost = build_cost(&cfgs[k]);
            jobs[k].index = k;
        }
        qsort(jobs, count, sizeof(build_job), cmp_build_job);
#pragma omp parallel for schedule(dynamic, 1)
        for (size_t q = 0; q < count; ++q) {
            const size_t k = jobs[q].index;
            sp_dev_use_device(dev);
            int r = model_from_config(&cfgs[k], &ms[k]);
            if (!r)
                r = sp_model_build_seeded(&ms[k], seeds[k]);
            rcs[k] = r;
        }
        for (size_t k = 0; k < count && !rc; ++k)
            rc = rcs[k];
        free(rcs);
        free(jobs);
    } else {
        /* one global rand() sequence, as count consecutive creates */
        for (size_t k = 0; k < count && !rc; ++k) {
            rc = model_from_config(&cfgs[k], &ms[k]);
            if (!rc)
                rc = sp_model_build(&ms[k]);
        }
    }
    const double t1 = now_ms();
    if (!rc)
        rc = sp_batch_create(ms, count, &h->b);
    h->construct_ms = t1 - t0;
    h->setup_ms = now_ms() - t1;
    if (rc) {
        for (size_t k = 0; k < count; ++k)
            sp_model_free(&ms[k]); /* no-op on zeroed or never-built entries */
        free(ms);
        free(h);
        return to_status(rc);
    }
    free(ms);
    h->count = count;
    *out = h;
    return SPIRES_OK;
}

SPIRES_EXPORT void spires_ext_batch_destroy(spires_ext_batch *b)
{
    if (!b)
        return;
    sp_batch_destroy(b->b);
    free(b);
}

SPIRES_EXPORT spires_status spires_ext_batch_run(spires_ext_batch *b, const double *const *u,
                                                 const size_t *T, uint32_t *const *rasters,
                                                 double *const *final_states,
                                                 double *elapsed_ms)
{
    if (!b || !T)
        return SPIRES_ERR_INVALID_ARG;
    return to_status(sp_batch_run(b->b, u, T, rasters, final_states, elapsed_ms));
}

SPIRES_EXPORT spires_status spires_ext_batch_train_ridge(spires_ext_batch *b,
                                                         const double *const *u,
                                                         const double *const *y,
                                                         const size_t *T, const double *lambda,
                                                         const spires_ext_ridge_opts *opts,
                                                         double *const *w_out,
                                                         double *elapsed_ms)
{
    if (!b || !T || !y || !lambda)
        return SPIRES_ERR_INVALID_ARG;
    sp_ridge_opts o;
    memset(&o, 0, sizeof(o));
    o.gram_mode = SPIRES_EXT_GRAM_FP64;
    o.max_refine = 30;
    o.refine_tol = 1e-13;
    if (opts) {
        o.gram_mode = opts->gram_mode;
        o.max_refine = opts->max_refine;
        o.refine_tol = opts->refine_tol;
        o.washout = opts->washout;
        o.gram_slices = opts->gram_slices;
    }
    for (size_t k = 0; k < b->count; ++k)
        if (!y[k] || o.washout >= T[k])
            return SPIRES_ERR_INVALID_ARG;
    return to_status(sp_batch_train_ridge(b->b, u, y, T, lambda, &o, w_out, elapsed_ms));
}

SPIRES_EXPORT spires_status spires_ext_batch_predict(spires_ext_batch *b, const double *const *u,
                                                     const size_t *T, double *const *y,
                                                     double *elapsed_ms)
{
    if (!b || !T)
        return SPIRES_ERR_INVALID_ARG;
    return to_status(sp_batch_predict(b->b, u, T, y, elapsed_ms));
}

SPIRES_EXPORT spires_status spires_ext_batch_fit_predict(
    spires_ext_batch *b, const double *const *u, const double *const *y, const size_t *T,
    const size_t *T_fit, const double *lambda, const spires_ext_ridge_opts *opts,
    double *const *y_out, double *const *w_out, double *elapsed_ms)
{
    if (!b || !T || !T_fit || !y || !lambda)
        return SPIRES_ERR_INVALID_ARG;
    sp_ridge_opts o;
    memset(&o, 0, sizeof(o));
    o.gram_mode = SPIRES_EXT_GRAM_FP64;
    o.max_refine = 30;
    o.refine_tol = 1e-13;
    if (opts) {
        o.gram_mode = opts->gram_mode;
        o.max_refine = opts->max_refine;
        o.refine_tol = opts->refine_tol;
        o.washout = opts->washout;
        o.gram_slices = opts->gram_slices;
    }
    for (size_t k = 0; k < b->count; ++k)
        if (!y[k] || T_fit[k] > T[k] || o.washout >= T_fit[k])
            return SPIRES_ERR_INVALID_ARG;
    return to_status(
        sp_batch_fit_predict(b->b, u, y, T, T_fit, lambda, &o, y_out, w_out, elapsed_ms));
}

SPIRES_EXPORT spires_status spires_ext_batch_autotune(spires_ext_batch *b,
                                                     const double *const *u, const size_t *T,
                                                     int *schedule, int *ctas, double *best_ms)
{
    if (!b || !T)
        return SPIRES_ERR_INVALID_ARG;
    for (size_t k = 0; k < b->count; ++k)
        if (T[k] == 0)
            return SPIRES_ERR_INVALID_ARG;
    return to_status(sp_batch_autotune(b->b, u, T, schedule, ctas, best_ms));
}

SPIRES_EXPORT spires_status spires_ext_batch_info(const spires_ext_batch *b, int *ctas,
                                                  int *groups, int *graph)
{
    if (!b)
        return SPIRES_ERR_INVALID_ARG;
    return to_status(sp_batch_info(b->b, ctas, groups, graph));
}

SPIRES_EXPORT spires_status spires_ext_spectral_radius(size_t n, const int64_t *row_ptr,
                                                       const int32_t *col, const double *w,
                                                       int on_device, double *out)
{
    if (!row_ptr || !out || (row_ptr[n] > 0 && (!col || !w)))
        return SPIRES_ERR_INVALID_ARG;
    if (on_device)
        return to_status(sp_dev_spectral_radius(n, row_ptr, col, w, out));
    *out = sp_csr_spectral_radius(n, row_ptr, col, w);
    return SPIRES_OK;
}

SPIRES_EXPORT spires_status spires_ext_model_build_seeded(const spires_reservoir_config *cfg,
                                                          unsigned seed, spires_ext_model **out)
{
    if (!cfg || !out)
        return SPIRES_ERR_INVALID_ARG;
    spires_ext_model *h = calloc(1, sizeof(*h));
    if (!h)
        return SPIRES_ERR_ALLOC;
    int rc = model_from_config(cfg, &h->m);
    h->m.host_only = 1;
    if (!rc)
        rc = sp_model_build_seeded(&h->m, seed);
    if (rc) {
        sp_model_free(&h->m);
        free(h);
        return to_status(rc);
    }
    *out = h;
    return SPIRES_OK;
}

/* ---- surrogate MLP ---------------------------------------------------------- */
struct spires_ext_mlp {
    sp_mlp *m;
};

SPIRES_EXPORT size_t spires_ext_mlp_num_params(void) { return (size_t)sp_mlp_num_params(); }

SPIRES_EXPORT spires_status spires_ext_mlp_create(uint64_t seed, spires_ext_mlp **out)
{
    if (!out)
        return SPIRES_ERR_INVALID_ARG;
    *out = NULL;
    spires_ext_mlp *h = calloc(1, sizeof(*h));
    if (!h)
        return SPIRES_ERR_ALLOC;
    int rc = sp_mlp_create(seed, &h->m);
    if (rc) {
        free(h);
        return to_status(rc);
    }
    *out = h;
    return SPIRES_OK;
}

SPIRES_EXPORT void spires_ext_mlp_destroy(spires_ext_mlp *m)
{
    if (!m)
        return;
    sp_mlp_destroy(m->m);
    free(m);
}

SPIRES_EXPORT spires_status spires_ext_mlp_get_params(spires_ext_mlp *m, float *params)
{
    if (!m || !params)
        return SPIRES_ERR_INVALID_ARG;
    return to_status(sp_mlp_get_params(m->m, params));
}

SPIRES_EXPORT spires_status spires_ext_mlp_set_params(spires_ext_mlp *m, const float *params)
{
    if (!m || !params)
        return SPIRES_ERR_INVALID_ARG;
    return to_status(sp_mlp_set_params(m->m, params));
}

SPIRES_EXPORT spires_status spires_ext_mlp_loss_grad(spires_ext_mlp *m, const float *X,
                                                     const float *y, size_t n, float *loss,
                                                     float *grad)
{
    if (!m || !X || !y || !loss || n == 0 || n > 1u << 24)
        return SPIRES_ERR_INVALID_ARG;
    return to_status(sp_mlp_loss_grad(m->m, X, y, (int)n, loss, grad));
}

SPIRES_EXPORT spires_status spires_ext_mlp_train(spires_ext_mlp *m, const float *X, const float *y,
                                                 size_t n, int epochs, int batch, float lr,
                                                 uint64_t seed, float *final_loss)
{
    if (!m || !X || !y || n == 0 || n > 1u << 24)
        return SPIRES_ERR_INVALID_ARG;
    return to_status(sp_mlp_train(m->m, X, y, (int)n, epochs, batch, lr, seed, final_loss));
}

SPIRES_EXPORT spires_status spires_ext_mlp_predict(spires_ext_mlp *m, const float *X, size_t n,
                                                   int bf16, float *mean, float *logvar)
{
    if (!m || !X || n == 0 || n > 1u << 24)
        return SPIRES_ERR_INVALID_ARG;
    return to_status(sp_mlp_predict(m->m, X, (int)n, bf16, mean, logvar));
}

SPIRES_EXPORT long long spires_ext_mlp_kernel_launches(const spires_ext_mlp *m)
{
    return m ? sp_mlp_launches(m->m) : 0;
}

SPIRES_EXPORT spires_status spires_ext_ridge_fit(const double *states, size_t T, size_t n,
                                                 const double *targets, size_t dout,
                                                 double lambda,
                                                 const spires_ext_ridge_opts *opts,
                                                 double *w_out, spires_ext_ridge_report *report)
{
    if (!states || !targets || !w_out || n == 0 || n > (size_t)INT32_MAX || dout == 0 ||
        dout > (size_t)INT32_MAX)
        return SPIRES_ERR_INVALID_ARG;
    sp_ridge_opts o;
    memset(&o, 0, sizeof(o));
    o.gram_mode = sp_default_gram_mode();
    o.max_refine = 30;
    o.refine_tol = 1e-13;
    if (opts) {
        o.gram_mode = opts->gram_mode;
        o.max_refine = opts->max_refine;
        o.refine_tol = opts->refine_tol;
        o.washout = opts->washout;
        o.gram_slices = opts->gram_slices;
    }
    if (o.washout >= T)
        return SPIRES_ERR_INVALID_ARG;
    sp_ridge_report rep;
    int rc = sp_ridge_host(states, T, (int)n, targets, (int)dout, lambda, &o, &rep, w_out);
    if (report) {
        report->gram_mode_used = rep.gram_mode_used;
        report->refine_iters = rep.refine_iters;
        report->rel_residual = rep.rel_residual;
        report->collect_ms = rep.collect_ms;
        report->gram_ms = rep.gram_ms;
        report->factor_ms = rep.factor_ms;
        report->refine_ms = rep.refine_ms;
        report->factor_failed = rep.factor_failed;
        report->lu_fallback = rep.lu_fallback;
        report->dual = rep.dual;
        report->solve_ms = rep.solve_ms;
    }
    if (rc == SP_RIDGE_SINGULAR)
        return SPIRES_ERR_INTERNAL;
    return to_status(rc);
}

SPIRES_EXPORT spires_status spires_ext_batch_timing(const spires_ext_batch *b, double *construct_ms,
                                                    double *setup_ms)
{
    if (!b)
        return SPIRES_ERR_INVALID_ARG;
    if (construct_ms)
        *construct_ms = b->construct_ms;
    if (setup_ms)
        *setup_ms = b->setup_ms;
    return SPIRES_OK;
}

/* The arrays of a model that a change of recurrent weights rebuilds: freed
 * (do_free) or just forgotten, when another copy of the model owns them. */
static void drop_graph_arrays(sp_host_model *m, int do_free)
{
    void *p[] = {m->row_ptr, m->col, m->w, m->edge_decay, m->edge_omd, m->edge_tau,
                 m->syn_coef, m->mexp_decay, m->mexp_omd, m->mexp_c, m->mexp_tau};
    if (do_free)
        for (size_t k = 0; k < sizeof(p) / sizeof(p[0]); ++k)
            free(p[k]);
    m->row_ptr = NULL;
    m->col = NULL;
    m->w = NULL;
    m->edge_decay = m->edge_omd = m->edge_tau = m->syn_coef = NULL;
    m->mexp_decay = m->mexp_omd = m->mexp_c = m->mexp_tau = NULL;
}

/* Replace the recurrent weights by a dense matrix (zeros are no edge), as the
 * reference's synapse_build_from_dense builds them (per-edge synapse draws
 * included), optionally rescaled to the configured spectral radius with the
 * construction's power iteration; the reservoir returns to its reset state.
 * The new graph is built beside the old one, which stays in place (host and
 * device) if anything fails. */
SPIRES_EXPORT spires_status spires_ext_set_weights(spires_reservoir *r, const double *dense,
                                                   int rescale)
{
    if (!r || !r->dev || !dense)
        return SPIRES_ERR_INVALID_ARG;
    sp_host_model t = r->m; /* shares the neuron-side arrays with r->m */
    drop_graph_arrays(&t, 0);
    int rc = sp_model_set_dense_weights(&t, dense);
    if (!rc && rescale) {
        double sr = 0.0;
        if (t.nnz < ((size_t)1 << 15) ||
            sp_dev_spectral_radius(t.n, t.row_ptr, t.col, t.w, &sr) != SP_OK)
            sr = sp_csr_spectral_radius(t.n, t.row_ptr, t.col, t.w);
        t.spectral_radius_before = sr;
        if (sr > 1e-9) {
            const double f = t.spectral_radius / sr;
            for (size_t k = 0; k < t.nnz; k++)
                t.w[k] = f * t.w[k];
        }
    }
    if (!rc)
        rc = sp_model_derive_neuron(&t);
    sp_dev *nd = NULL;
    if (!rc)
        rc = sp_dev_create(&t, &nd);
    if (rc) {
        drop_graph_arrays(&t, 1);
        return to_status(rc);
    }
    drop_graph_arrays(&r->m, 1);
    r->m = t;
    sp_dev_destroy(r->dev);
    r->dev = nd;
    return SPIRES_OK;
}
