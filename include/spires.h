/*
 * spires.h -- public C API of the B200 spires library.
 *
 * Drop-in replacement for txmastin/spires `include/spires.h`: every type,
 * enumerator value, struct layout and function signature below is identical to
 * the reference header (include/spires.h:25-267 upstream), so programs built
 * against the reference relink against this library unchanged. The
 * implementation behind it runs the reservoir dynamics and readouts as CUDA
 * kernels on one NVIDIA B200 (sm_100a); construction stays on the host so the
 * weights match the reference draw for draw from the C library's rand().
 *
 * Conventions kept from the reference:
 *   - opaque handle, status codes, snake_case;
 *   - neuron_params / synapse_params are owned by the caller and are read
 *     again by spires_reservoir_reset (the pointer is kept, not the values);
 *   - buffers returned by spires_run / spires_copy_* come from malloc() and
 *     are released by the caller with free();
 *   - spires_step / spires_run / spires_read_* allocate no device memory:
 *     everything the dynamics need is sized at create time.
 *
 * Differences (documented, all on paths where the reference crashes or exits):
 *   - spires_step(r, NULL) steps with a zero input vector as documented
 *     (the reference dereferences NULL);
 *   - an unknown neuron/synapse/topology enumerator makes create return
 *     SPIRES_ERR_INVALID_ARG (the reference calls exit());
 *   - CUDA failures map to SPIRES_ERR_INTERNAL, device allocation failures to
 *     SPIRES_ERR_ALLOC.
 */
#ifndef SPIRES_H
#define SPIRES_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
typedef enum {
    SPIRES_OK = 0,
    SPIRES_ERR_INVALID_ARG,
    SPIRES_ERR_ALLOC,
    SPIRES_ERR_INTERNAL
} spires_status;

/* Opaque reservoir handle. */
typedef struct spires_reservoir spires_reservoir;

/* Recurrent topology. */
typedef enum {
    SPIRES_CONN_RANDOM = 0,     /* Erdos-Renyi, edge probability = connectivity */
    SPIRES_CONN_SMALL_WORLD,    /* Watts-Strogatz ring, K = round(c (n-1)), p = 0.1 */
    SPIRES_CONN_SCALE_FREE      /* Barabasi-Albert, m = round(c (n-1)), random orientation */
} spires_connectivity_type;

/* Neuron model (neuron_params layout in brackets). */
typedef enum {
    SPIRES_NEURON_LIF_DISCRETE = 0, /* [V_0, V_th, leak_rate, bias] */
    SPIRES_NEURON_LIF_BIO,          /* [V_0, V_th, tau, bias] */
    SPIRES_NEURON_FLIF_CAPUTO,      /* [C_m, g_l, V_l, V_th, V_reset, V_peak, alpha, t_ref, T_mem] */
    SPIRES_NEURON_FLIF_GL,          /* [V_th, V_reset, V_rest, tau_m, alpha, T_mem, bias, t_ref] */
    SPIRES_NEURON_FLIF_DIFFUSIVE    /* [V_th, V_reset, V_rest, tau_m, alpha, T_mem_or_tref, bias] */
} spires_neuron_type;

/* Synapse model of the recurrent connections (synapse_params layout):
 *   SIMPLE              unused; input = sum_j w_ij spike_j
 *   PSC_HOMOGENEOUS     [tau_syn]; one exponential trace per presynaptic neuron
 *   PSC_HETEROGENEOUS   [tau_min, tau_max]; per-edge tau, log-uniform
 *   FRACTIONAL          [alpha, tau_syn, T_mem]; Grunwald-Letnikov fractional
 *                       relaxation of the synaptic current per neuron
 *   FRACTIONAL_MULTIEXP [alpha, tau_syn, tau_min, tau_max, N]; sum of N
 *                       exponential traces weighted by the Mittag-Leffler
 *                       spectral density
 */
typedef enum {
    SPIRES_SYNAPSE_SIMPLE = 0,
    SPIRES_SYNAPSE_PSC_HOMOGENEOUS,
    SPIRES_SYNAPSE_PSC_HETEROGENEOUS,
    SPIRES_SYNAPSE_FRACTIONAL,
    SPIRES_SYNAPSE_FRACTIONAL_MULTIEXP
} spires_synapse_type;

/* Storage of the recurrent weights. Both produce bit-identical dynamics here
 * (a zero weight contributes an exact zero to a sum that starts at +0). */
typedef enum {
    SPIRES_SYNAPSE_SPARSE = 0,
    SPIRES_SYNAPSE_DENSE
} spires_synapse_backend;

/* Creation-time configuration. */
typedef struct {
    size_t num_neurons;
    size_t num_inputs;
    size_t num_outputs;
    double spectral_radius;
    double ei_ratio;
    double input_strength;
    double connectivity;
    double dt;                                 /* micro-step; 1/dt must be an integer */
    spires_connectivity_type connectivity_type;
    spires_neuron_type       neuron_type;
    double *neuron_params;                     /* caller owns; kept by pointer */
    spires_synapse_type      synapse_type;     /* 0 = SIMPLE */
    spires_synapse_backend   synapse_backend;  /* 0 = SPARSE */
    double *synapse_params;                    /* caller owns; kept by pointer */
} spires_reservoir_config;

/* ---- lifecycle ---- */
/* replaces reference include/spires.h:131, src/spires_api.c:22-75 */
spires_status spires_reservoir_create(const spires_reservoir_config *cfg,
                                      spires_reservoir **out_r);
/* include/spires.h:133, src/spires_api.c:77-84 */
void          spires_reservoir_destroy(spires_reservoir *r);
/* include/spires.h:134, src/spires_api.c:86-92 */
spires_status spires_reservoir_reset(spires_reservoir *r);

/* ---- stepping ---- */
/* One macro step (1/dt micro-steps) with input u_t[num_inputs]; NULL = zeros.
 * include/spires.h:142, src/spires_api.c:95-102 */
spires_status spires_step(spires_reservoir *r, const double *u_t);

/* Run input_series[series_length x num_inputs]; returns a malloc'd
 * [series_length x num_outputs] array of readouts (caller frees), or NULL.
 * include/spires.h:155, src/spires_api.c:106-112 */
double *spires_run(spires_reservoir *r, const double *input_series, size_t series_length);

/* ---- training ----
 * include/spires.h:161-177; src/spires_api.c:117-154 (online, ridge, RLS),
 * src/spires_api.c:226-245 (coarse-grain) */
spires_status spires_train_online(spires_reservoir *r,
                                  const double *target_vec, double lr);

spires_status spires_train_ridge(spires_reservoir *r,
                                 const double *input_series,
                                 const double *target_series,
                                 size_t series_length, double lambda);

spires_status spires_train_rls(spires_reservoir *r,
                               const double *input_series,
                               const double *target_series,
                               size_t series_length,
                               double delta, double lambda);

spires_status spires_coarse_grain(const spires_reservoir *r,
                                  double weight_threshold,
                                  spires_reservoir **out_r);

/* ---- state access ----
 * include/spires.h:185-218; src/spires_api.c:157-223 */
double       *spires_copy_reservoir_state(spires_reservoir *r);          /* malloc'd [N] */
spires_status spires_read_reservoir_state(spires_reservoir *r, double *buffer);
spires_status spires_read_spike_state(spires_reservoir *r, double *buffer); /* 0.0 / 1.0 */
double       *spires_copy_weights(const spires_reservoir *r);            /* malloc'd [N*N] */
spires_status spires_read_weights(const spires_reservoir *r, double *buffer);
spires_status spires_compute_output(spires_reservoir *r, double *out);   /* y = W_out V */
double       *spires_copy_readout(const spires_reservoir *r);            /* malloc'd [Dout*N] */
spires_status spires_read_readout(const spires_reservoir *r, double *buffer);

/* ---- introspection ---- include/spires.h:226-228, src/spires_api.c:248-261 */
size_t spires_num_neurons(const spires_reservoir *r);
size_t spires_num_inputs(const spires_reservoir *r);
size_t spires_num_outputs(const spires_reservoir *r);

/* ---- hyper-parameter search (AGILE) ----
 * include/spires.h:235-267, src/spires_api.c:440-498 */
struct spires_opt_budget {
    double data_fraction;    /* 0..1 */
    int    num_seeds;
    double time_limit_sec;   /* 0 = no limit */
    int    _reserved_i0;
    double _reserved_d0;
};

enum spires_metric_kind { SPIRES_METRIC_AUROC = 0, SPIRES_METRIC_AUPRC = 1 };

struct spires_opt_score {
    double lambda_var;       /* penalty on std(metric) */
    double lambda_cost;      /* penalty on the cost proxy */
    int    metric;           /* enum spires_metric_kind */
    int    _reserved_i0;
};

struct spires_opt_result {
    spires_reservoir_config best_config;
    double                  best_log10_ridge;
    double                  best_score;   /* mean - lambda_var*std - lambda_cost*cost */
    double                  metric_mean;
    double                  metric_std;
};

int spires_optimize(const spires_reservoir_config *base_config,
                    const struct spires_opt_budget *budgets,
                    int num_budgets,
                    const struct spires_opt_score *score,
                    struct spires_opt_result *out,
                    const double *input_series,
                    const double *target_series,
                    size_t series_length);

#ifdef __cplusplus
} /* extern "C" */
#endif
#endif /* SPIRES_H */
