/*
 * sp_model.h -- host-side reservoir model shared by the C host code and the
 * CUDA layer (plain C types only; no CUDA or torch types cross this header).
 *
 * A model is built on the host exactly as the reference builds it
 * (src/reservoir.c:345-571, src/synapse.c:3-30, src/synapses/<type>.c build
 * functions), consuming the C library's rand() in the same order, and every
 * constant the reference obtains from libm (pow, exp, log, tgamma, sin, cos)
 * is evaluated here with the host libm and handed to the device as bits. The
 * device kernels therefore only add, subtract, multiply and divide in IEEE
 * double with round-to-nearest and no contraction.
 */
#ifndef SP_MODEL_H
#define SP_MODEL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { SP_LIF_DISCRETE = 0, SP_LIF_BIO, SP_FLIF_CAPUTO, SP_FLIF_GL, SP_FLIF_DIFFUSIVE };
enum { SP_SYN_SIMPLE = 0, SP_SYN_PSC_HOM, SP_SYN_PSC_HET, SP_SYN_FRAC, SP_SYN_FRAC_MEXP };
enum { SP_CONN_RANDOM = 0, SP_CONN_SMALL_WORLD, SP_CONN_SCALE_FREE };

/* Upper bound on ring lengths, as in the reference (flif_gl.h:4,
 * flif_caputo.h:4, synapses/fractional.c:7). */
#define SP_MAX_MEM_LEN 20000

/* Per-model scalar parameters, derived on the host from neuron_params. */
typedef struct {
    /* LIF_DISCRETE: a = V_0, b = V_th, c = (1 - leak_rate), d = bias
     * LIF_BIO:      a = V_0, b = V_th, c = tau,            d = bias
     * FLIF_GL:      a = V_th, b = V_reset, c = V_rest, d = tau_m, e = bias,
     *               f = t_ref, g = dt^alpha
     * FLIF_CAPUTO:  a = V_th, b = V_0, c = g_l, d = V_l, e = C_m, f = t_ref,
     *               g = kr = dt^alpha * Gamma(2 - alpha)
     * FLIF_DIFFUSIVE: a = V_th, b = V_reset, c = V_rest, d = bias,
     *               e = g_euler = dt / tau_m, f = t_min, g = t_max, h = t_ref,
     *               i = m = alpha^2, j = q = 6 alpha, k = tmin^(1-q), l = tmax^(1-q)
     */
    double a, b, c, d, e, f, g, h, i, j, k, l;
    double v_init;      /* membrane potential after init / reset */
    double tprev_init;  /* refractory clock after init / reset */
    int    L;           /* FLIF_GL ring length; FLIF_CAPUTO shift-register depth (mem_len-2) */
    int    det_refr_steps;  /* FLIF_DIFFUSIVE, alpha >= 1: ceil(t_ref/dt) */
    int    diff_stochastic; /* FLIF_DIFFUSIVE: alpha < 1 */
} sp_neuron_consts;

typedef struct {
    double decay, omd;          /* PSC_HOM: exp(-dt/tau), 1 - exp(-dt/tau) */
    double frac_dta, frac_tau;  /* FRACTIONAL: dt^alpha, tau_syn */
    int    frac_L;              /* FRACTIONAL ring length */
    int    mexp_N;              /* MULTIEXP component count */
} sp_synapse_consts;

typedef struct sp_host_model {
    /* configuration (the parameter arrays are caller-owned pointers) */
    size_t n, din, dout;
    double spectral_radius, ei_ratio, input_strength, connectivity, dt;
    int conn_type, neuron_type, syn_type, syn_backend;
    double *neuron_params;
    double *synapse_params;
    int micro_steps;

    /* weights */
    double  *W_in;     /* n x din, row-major */
    double  *W_out;    /* dout x n, row-major */
    int64_t *row_ptr;  /* n + 1 */
    int32_t *col;      /* nnz, ascending within each row */
    double  *w;        /* nnz */
    size_t   nnz;

    /* neuron constants */
    sp_neuron_consts nc;
    double *coef;      /* FLIF_GL: GL coefficients [L]; FLIF_CAPUTO: L1 weights [L] */

    /* synapse constants */
    sp_synapse_consts sc;
    double *edge_decay;  /* PSC_HET: exp(-dt/tau_k) per stored edge */
    double *edge_omd;    /* PSC_HET: 1 - exp(-dt/tau_k) */
    double *edge_tau;    /* PSC_HET: tau_k per stored edge */
    double *syn_coef;    /* FRACTIONAL: GL coefficients [frac_L] */
    double *mexp_decay;  /* MULTIEXP: [mexp_N] */
    double *mexp_omd;    /* MULTIEXP: [mexp_N] */
    double *mexp_c;      /* MULTIEXP: [mexp_N] mixing weights */
    double *mexp_tau;    /* MULTIEXP: [mexp_N] */

    /* diagnostics from construction */
    double spectral_radius_before;  /* power-iteration estimate before rescale */
    double topology_ms;             /* host time drawing the recurrent graph */
    double spectral_ms;             /* host time of the spectral-radius rescale */
    uint64_t diffusive_seed;        /* FLIF_DIFFUSIVE per-reservoir seed */

    /* construction policy: 1 = never use the GPU (spires_ext_model_build) */
    int host_only;
} sp_host_model;

/* status codes mirror spires_status */
enum { SP_OK = 0, SP_EINVAL = 1, SP_EALLOC = 2, SP_EINTERNAL = 3, SP_RIDGE_SINGULAR = 100 };

/* construct.c */
int  sp_validate_config(size_t n, size_t din, size_t dout, double dt, int conn_type,
                        int neuron_type, const double *neuron_params, int syn_type,
                        int syn_backend);
int  sp_model_build(sp_host_model *m);          /* fills weights, consumes rand() */
int  sp_model_derive_neuron(sp_host_model *m);  /* re-reads neuron_params (create and reset) */
void sp_model_free(sp_host_model *m);
/* Private generator with glibc's srand(seed) + rand() sequence (construct.c). */
typedef struct {
    int32_t r[31];
    int f, b;
} sp_rand_state;
void sp_rand_seed(sp_rand_state *s, unsigned seed);
int  sp_rand_next(sp_rand_state *s);

/* sp_model_build drawing from a private generator seeded with `seed` instead
 * of the global rand(): the same model as srand(seed) + sp_model_build, and
 * safe to run on several threads at once. */
int sp_model_build_seeded(sp_host_model *m, unsigned seed);

/* The same power iteration on the current CUDA device, bit-identical to
 * sp_csr_spectral_radius (dev_construct.cu); non-zero status = not done. */
int sp_dev_spectral_radius(size_t n, const int64_t *row_ptr, const int32_t *col,
                           const double *w, double *out);
double sp_csr_spectral_radius(size_t n, const int64_t *row_ptr, const int32_t *col,
                              const double *w);
int  sp_model_build_synapse(sp_host_model *m, const double *dense_or_null);
int  sp_model_set_dense_weights(sp_host_model *m, const double *dense);

#ifdef __cplusplus
}
#endif
#endif
