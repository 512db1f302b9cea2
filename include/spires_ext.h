/*
 * spires_ext.h -- additive entry points of the B200 spires library.
 *
 * Nothing here exists in the reference header; these calls carry what
 * spires.h cannot express (device-resident series, recorded state matrices,
 * spike rasters, mixed-precision ridge options, washout, host-only model
 * inspection) and the tuning hooks of the GPU implementation. All use plain C
 * types; device pointers are passed as `const double *` / `double *` and are
 * documented as such.
 */
#ifndef SPIRES_EXT_H
#define SPIRES_EXT_H

#include <stddef.h>
#include <stdint.h>
#include "spires.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- host-only model (no GPU needed) -------------------------------------
 * Runs the construction of spires_reservoir_create (same rand() draws, same
 * spectral-radius rescale) on the host and exposes the result. Used to check
 * construction against the reference on machines without a GPU. */
typedef struct spires_ext_model spires_ext_model;

typedef struct {
    size_t num_neurons, num_inputs, num_outputs, nnz;
    int    ring_len;          /* FLIF_GL history length L (Caputo: mem_len - 2) */
    int    micro_steps;       /* 1/dt */
    int    syn_ring_len;      /* FRACTIONAL synapse history length */
    int    syn_components;    /* FRACTIONAL_MULTIEXP component count */
    double spectral_radius_before_rescale;
    double topology_ms;       /* host time drawing the recurrent graph */
    double spectral_ms;       /* time of the spectral-radius rescale (host or device) */
} spires_ext_model_info;

spires_status spires_ext_model_build(const spires_reservoir_config *cfg,
                                     spires_ext_model **out);
/* As spires_ext_model_build after srand(seed), but drawing from a private
 * generator with the same sequence as glibc's srand(seed) + rand(): the global
 * rand() state is left alone and several threads may build at once. */
spires_status spires_ext_model_build_seeded(const spires_reservoir_config *cfg, unsigned seed,
                                            spires_ext_model **out);
void          spires_ext_model_free(spires_ext_model *m);
spires_status spires_ext_model_info_get(const spires_ext_model *m,
                                        spires_ext_model_info *info);
/* CSR of W (ascending columns); any pointer may be NULL */
spires_status spires_ext_model_csr(const spires_ext_model *m, int64_t *row_ptr,
                                   int32_t *col, double *val);
spires_status spires_ext_model_w_in(const spires_ext_model *m, double *w_in);
spires_status spires_ext_model_w_out(const spires_ext_model *m, double *w_out);
/* PSC_HETEROGENEOUS per-edge tau in CSR order */
spires_status spires_ext_model_edge_tau(const spires_ext_model *m, double *tau);
/* FLIF_GL / FLIF_CAPUTO coefficient table [ring_len] */
spires_status spires_ext_model_coef(const spires_ext_model *m, double *coef);

/* ---- recorded runs -------------------------------------------------------
 * Advance `T` macro steps from the current state with inputs u[T x num_inputs]
 * (host memory; NULL = zeros) and record, after every macro step, the state
 * (phi [T x N], may be NULL), the spike bits (raster [T x ceil(N/32)] words,
 * bit i%32 of word i/32 = neuron i, may be NULL) and the readout
 * (y [T x num_outputs], may be NULL). */
spires_status spires_ext_run_record(spires_reservoir *r, const double *u, size_t T,
                                    double *phi, uint32_t *raster, double *y);

/* Same, with every pointer in device memory (u may be NULL); asynchronous on
 * the handle's stream; completion and errors via spires_ext_sync. */
spires_status spires_ext_run_device(spires_reservoir *r, const double *d_u, size_t T,
                                    double *d_phi, uint32_t *d_raster, double *d_y);
spires_status spires_ext_sync(spires_reservoir *r);
void         *spires_ext_stream(spires_reservoir *r);    /* cudaStream_t */
size_t        spires_ext_spike_words(const spires_reservoir *r);
long long     spires_ext_kernel_launches(const spires_reservoir *r);

/* Input weights W_in [N x num_inputs] of a reservoir (host copy). */
spires_status spires_ext_read_w_in(const spires_reservoir *r, double *w_in);

/* ---- launch shape of the persistent step kernel --------------------------- */
typedef struct {
    int ctas;         /* CTAs of the cooperative grid; 1 = single CTA */
    int warps_max;    /* warps per CTA */
    int variant;      /* 0 = generic, 1 = bulk-copy ring pipeline (FLIF_GL) */
    int stages;       /* pipeline stages (variant 1) */
    int rows;         /* ring rows per stage (variant 1) */
    int csr_global;   /* 1: walk the recurrent CSR rows in global memory even
                         when the CTA's slice fits in shared memory (0 default) */
    int l2_pin;       /* variant 1: the oldest l2_pin lags of every step are
                         loaded with L2 evict-last priority and younger lags
                         and the ring writes with evict-first, so that part of
                         a ring larger than the L2 stays resident from step to
                         step; 0 = no cache hints, -1 = automatic (default: 70 %
                         of the L2 when the ring is larger than three quarters
                         of it, else 0) */
} spires_ext_launch;

spires_status spires_ext_get_launch(const spires_reservoir *r, spires_ext_launch *l);
/* Ring lags the current launch keeps L2-resident (l2_pin with -1 resolved;
 * 0 for variant 0 or without cache hints). */
int           spires_ext_l2_pin_rows(const spires_reservoir *r);
spires_status spires_ext_set_launch(spires_reservoir *r, const spires_ext_launch *l);
/* Time candidate launch shapes on this reservoir (state is saved and restored)
 * and keep the fastest. `steps` macro steps per candidate. */
spires_status spires_ext_autotune(spires_reservoir *r, size_t steps);

/* FLIF_DIFFUSIVE refractory sampler seed (per reservoir; neuron i gets a
 * stream derived from seed and i). Takes effect at the next reset. */
spires_status spires_ext_set_seed(spires_reservoir *r, uint64_t seed);

/* ---- bounded waits and failure paths ---------------------------------------
 * No counterpart in the reference, which prints or exits on internal errors.
 * Every wait inside the step kernel (the grid barrier between micro-steps, the
 * history pipeline's barriers) is bounded: when one runs out, the kernel
 * records an error code (1 = a wait ran out) and the micro-step, every CTA
 * returns at its next wait, in-flight copies are drained, and the call that
 * waited for the launch returns SPIRES_ERR_INTERNAL. The reservoir's state
 * is then undefined until spires_reservoir_reset; the device stays usable.
 *
 * set_wait_limit: the limit of those waits in milliseconds (default 2000,
 * at most 60000).
 * last_device_error: code and micro-step (counted from the reservoir's
 * creation or last reset) of the last such error, 0 if none.
 * test_withhold_arrival: test hook, one-shot. In the next launch, CTA `cta`
 * does not arrive at the grid barrier that opens micro-step `micro_step`
 * (counted from that launch's first micro-step, >= 1), so the others' wait
 * runs out as it would if a CTA had stopped. Ignored by single-CTA launches.
 * test_fail_device_alloc: test hook, process-wide. After `after` more device
 * allocations by this library the next one fails (as an out-of-memory
 * cudaMalloc would), then allocations succeed again; -1 clears it.
 * test_live_device_allocs: device allocations of this library not yet freed
 * (process-wide), to check that failed calls release what they allocated. */
spires_status spires_ext_set_wait_limit(spires_reservoir *r, double ms);
spires_status spires_ext_last_device_error(const spires_reservoir *r, int *code,
                                           long long *micro_step);
spires_status spires_ext_test_withhold_arrival(spires_reservoir *r, int cta,
                                               long long micro_step);
void          spires_ext_test_fail_device_alloc(long long after);
long long     spires_ext_test_live_device_allocs(void);

/* ---- state checkpoint -------------------------------------------------------
 * Everything a run continues from: membrane potentials, refractory clocks,
 * the FLIF_GL history ring or Caputo registers, the FLIF_DIFFUSIVE sampler
 * states, the latest spike words, synaptic drive and traces, the fractional
 * synapse history, the step counters -- and the readout W_out. Saving waits
 * for the steps already queued; buf_bytes must be at least
 * spires_ext_state_bytes(r). The buffer starts with a header holding the
 * sizes (neurons, inputs, outputs, ring lengths, edges), the micro-step count,
 * the models and a 64-bit hash of everything the dynamics read (dt, the
 * derived neuron and synapse constants, the recurrent weights and their
 * pattern, W_in, the history coefficients). Load accepts only a buffer of
 * exactly spires_ext_state_bytes(r) bytes whose header equals this
 * reservoir's, and checks all of it before touching the reservoir
 * (SPIRES_ERR_INVALID_ARG otherwise, reservoir unchanged): a reservoir built
 * from the same configuration and seed then continues bit for bit as the saved
 * one would have. If a device copy fails during a load (SPIRES_ERR_INTERNAL),
 * the reservoir's state is undefined until spires_reservoir_reset. The weights
 * W and W_in are not part of the buffer. No counterpart in the reference,
 * which has no state setter. */
size_t        spires_ext_state_bytes(spires_reservoir *r);
spires_status spires_ext_state_save(spires_reservoir *r, void *buf, size_t buf_bytes);
spires_status spires_ext_state_load(spires_reservoir *r, const void *buf, size_t buf_bytes);

/* ---- recurrent weights from a dense matrix ----------------------------------
 * Replaces W by dense[N x N] (row-major, zero = no edge) the way the
 * reference's synapse_build_from_dense builds a synapse matrix (per-edge
 * synapse quantities drawn again from rand() where the model has them);
 * with rescale = 1 the weights are scaled to the configured spectral radius by
 * the construction's power iteration. The reservoir returns to its reset
 * state; W_in and W_out are kept. For workloads whose weights are not the
 * generator's (for example N(0,1) weights on an Erdos-Renyi pattern). */
spires_status spires_ext_set_weights(spires_reservoir *r, const double *dense, int rescale);

/* ---- spectral radius ------------------------------------------------------
 * The max-abs normalised power iteration that scales the recurrent weights at
 * create time (reference src/sparse.c:93-127) on an n x n CSR matrix with
 * ascending columns: on the current CUDA device (on_device = 1) or on the
 * host (0). Both give the same bits; spires_reservoir_create uses the device
 * for matrices with at least 2^15 edges unless SPIRES_HOST_SPECTRAL_RADIUS=1. */
spires_status spires_ext_spectral_radius(size_t n, const int64_t *row_ptr, const int32_t *col,
                                         const double *w, int on_device, double *out);

/* ---- ridge readout with options ------------------------------------------ */
/* The Gram X^T X of the fitted states (the reference forms it with one
 * cblas_dgemm, src/math_utils.c:154-162) in one of four ways; X^T Y, the
 * factorisation and the refinement residuals are FP64 in every mode. */
typedef enum {
    SPIRES_EXT_GRAM_FP64 = 0,      /* FP64 Gram (CUDA cores) */
    SPIRES_EXT_GRAM_BF16X3 = 1,    /* BF16 hi/lo split on the tensor cores
                                      (hi hi + hi lo + lo hi), FP32 accumulate;
                                      solved by Cholesky-preconditioned CG on
                                      the FP64 operator */
    SPIRES_EXT_GRAM_TF32X3 = 2,    /* the same with TF32 hi/lo */
    SPIRES_EXT_GRAM_INT8 = 3       /* error-free integer slices on the tensor
                                      cores (int8 digits, exact int32 sums per
                                      digit level, FP64 combination): a Gram as
                                      accurate as the FP64 one with 7 slices,
                                      then FP64 Cholesky and refinement */
} spires_ext_gram_mode;

typedef struct {
    int    gram_mode;        /* spires_ext_gram_mode */
    int    max_refine;       /* iterative-refinement sweeps */
    double refine_tol;       /* relative residual target */
    size_t washout;          /* leading rows excluded from the fit */
    int    gram_slices;      /* SPIRES_EXT_GRAM_INT8: slices, 2..8 (0 = 7) */
} spires_ext_ridge_opts;

typedef struct {
    int    gram_mode_used;
    int    refine_iters;
    double rel_residual;     /* ||Phi^T Y - (Phi^T Phi + lambda I) W|| / ||Phi^T Y|| */
    double collect_ms, gram_ms, factor_ms, refine_ms;
    int    factor_failed;
    int    lu_fallback;
    int    dual;             /* 1: fewer fitted rows than N/2, solved as
                                W = Phi^T (Phi Phi^T + lambda I)^-1 Y */
    double solve_ms;         /* the first triangular solve; factor_ms is the
                                factorisation alone */
} spires_ext_ridge_report;

/* The Gram C = X^T X (d_C [n x n], full matrix) of device states
 * d_X [T x n] over rows [t0, T) in any spires_ext_gram_mode (slices: the
 * INT8 mode's slice count, 0 = 7); `stream` is a cudaStream_t (NULL = default);
 * returns once the work on it has finished. Work memory is allocated on the
 * device (stream-ordered) and freed before the call returns. */
spires_status spires_ext_gram_device(const double *d_X, size_t T, size_t n, size_t t0,
                                     int mode, int slices, double *d_C, void *stream);

spires_status spires_ext_train_ridge(spires_reservoir *r, const double *input_series,
                                     const double *target_series, size_t series_length,
                                     double lambda, const spires_ext_ridge_opts *opts,
                                     spires_ext_ridge_report *report);

/* Ridge on states the caller already holds (host arrays): states [T x n]
 * row-major, targets [T x dout], rows [washout, T) fitted; w_out [dout x n].
 * The reservoir readouts' solver, including the dual form when fewer than
 * n/2 rows are fitted (the classification workload's 500 time-averaged
 * states against 20000 neurons) and the split-Gram modes; any number of
 * outputs (solved 16 at a time over one system matrix). A singular system
 * returns SPIRES_ERR_INTERNAL. */
spires_status spires_ext_ridge_fit(const double *states, size_t T, size_t n,
                                   const double *targets, size_t dout, double lambda,
                                   const spires_ext_ridge_opts *opts, double *w_out,
                                   spires_ext_ridge_report *report);

/* ---- AGILE search core ----------------------------------------------------
 * The black-box optimiser behind spires_optimize (reference src/agile.h:21-91,
 * same option and report layouts): Levy-step exploration with SPSA gradients,
 * then SPSA gradient-descent refinement, minimising loss(theta) within
 * [lower, upper]. Exposed so callers can tune their own objectives. */
typedef struct {
    double   mu, eta_min, eta_max, patience0, patience_decay;
    double   refine_step;
    int      refine_max_iters, refine_no_improve;
    double   spsa_eps;
    int      reflect_at_bounds;
    uint64_t seed;
    int      verbose;
} spires_ext_agile_opts;

typedef struct {
    double best_loss;
    int    best_iter, total_evals, total_iters, exited_refinement;
} spires_ext_agile_report;

typedef double (*spires_ext_loss_fn)(const double *theta, int dim, void *ctx);

spires_status spires_ext_agile_minimize(const double *theta0, const double *lower,
                                        const double *upper, int dim,
                                        spires_ext_loss_fn loss, void *ctx,
                                        const spires_ext_agile_opts *opts, double *theta_best,
                                        spires_ext_agile_report *report);

/* AGILE in ask/tell form for batched evaluation: `chains` independent
 * chains (start points theta0[chains][dim], one seed each, or opts->seed for
 * all when seeds is NULL) advanced in lockstep. ask writes the points every
 * live chain needs next (at most 2 * chains rows of dim, chain index of each
 * row in owner) and returns their count, 0 when every chain has finished;
 * tell takes their losses in the same order. Each chain visits exactly the
 * points spires_ext_agile_minimize visits with the same options and seed. */
typedef struct spires_ext_agile_batch spires_ext_agile_batch;

spires_status spires_ext_agile_batch_create(int chains, int dim, const double *theta0,
                                            const double *lower, const double *upper,
                                            const spires_ext_agile_opts *opts,
                                            const uint64_t *seeds,
                                            spires_ext_agile_batch **out);
void          spires_ext_agile_batch_destroy(spires_ext_agile_batch *b);
int           spires_ext_agile_batch_ask(spires_ext_agile_batch *b, double *points, int *owner);
spires_status spires_ext_agile_batch_tell(spires_ext_agile_batch *b, const double *losses);
spires_status spires_ext_agile_batch_best(const spires_ext_agile_batch *b, int chain,
                                          double *theta, spires_ext_agile_report *report);

/* ---- ridge readout without device allocation -----------------------------
 * No counterpart in the reference. For callers that cannot allocate device
 * memory themselves -- a host framework that owns every device buffer through
 * its own allocator or quota, or a control loop that cannot afford the
 * implicit device-wide synchronisation of cudaMalloc/cudaFree -- this solves
 * W_out = (X^T X + lambda I)^-1 X^T Y for states X = d_states[T][n] (rows
 * washout..T-1 used) and targets Y = d_targets[T][dout], both already in
 * device memory, and writes d_w_out[dout][n] (the spires_read_readout
 * layout). FP64 Gram, Cholesky and iterative refinement: the same kernels, in
 * the same order, as spires_ext_train_ridge with SPIRES_EXT_GRAM_FP64.
 * It calls no cudaMalloc/cudaFree: its working memory is one fixed array of
 * this library (8.6 MB, held on every GPU that loads the library until the
 * process exits), which bounds the sizes: n <= 512, dout <= 16, T <= 16384;
 * larger requests return SPIRES_ERR_INVALID_ARG. A singular system (the
 * Cholesky factorisation fails and so does LU with partial pivoting) returns
 * SPIRES_ERR_INTERNAL with d_w_out left as it was. The first call on a device
 * looks up the array's device address, so make that first call before any
 * stream capture. Every call shares the one array, so calls that overlap on
 * the GPU (other streams, other host threads) race; serialise them. `stream`
 * is a cudaStream_t (NULL = default stream). Each call waits on the host for
 * its work on that stream: the refinement reads a residual norm back after
 * every sweep, and the call returns after the last kernel has finished. */
spires_status spires_ext_ridge_solve_noalloc(const double *d_states, const double *d_targets,
                                             size_t T, size_t n, size_t dout, size_t washout,
                                             double lambda, double *d_w_out, void *stream);

/* ---- many reservoirs in one launch ---------------------------------------
 * No counterpart in the reference (its unit of work is one reservoir). A batch
 * holds `count` reservoirs of uneven size, ring length, series length and
 * model; instance k is built exactly as spires_reservoir_create builds it
 * after srand(seeds[k]), so its weights, and its spike rasters and states from
 * reset, are bit-identical to those of a separately created reservoir. With
 * seeds, the instances are built on all host threads from private generators
 * with glibc's srand/rand sequence and the global rand() state is untouched;
 * seeds = NULL draws every instance from the global rand() in turn.
 * Supported: SPIRES_NEURON_LIF_DISCRETE and SPIRES_NEURON_FLIF_GL with
 * SPIRES_SYNAPSE_SIMPLE, num_outputs <= 16; anything else returns
 * SPIRES_ERR_INVALID_ARG. Every call starts all instances from their reset
 * state. Series arrays are indexed by instance: u[k] is T[k] x num_inputs_k
 * (NULL array or NULL entry = zeros). The whole batch runs as one persistent
 * cooperative kernel (one CUDA graph replay while the series lengths stay the
 * same), so one call costs one launch sequence however many instances it has. */
typedef struct spires_ext_batch spires_ext_batch;

spires_status spires_ext_batch_create(const spires_reservoir_config *cfgs,
                                      const unsigned *seeds, size_t count,
                                      spires_ext_batch **out);
void          spires_ext_batch_destroy(spires_ext_batch *b);

/* Spike rasters (T[k] x ceil(N_k/32) words, bit i%32 of word i/32 = neuron i)
 * and final membrane states (N_k) of every instance; NULL entries skip an
 * output. elapsed_ms (optional): device time of the launch sequence. */
spires_status spires_ext_batch_run(spires_ext_batch *b, const double *const *u,
                                   const size_t *T, uint32_t *const *rasters,
                                   double *const *final_states, double *elapsed_ms);

/* Ridge readout of every instance (FP64, as spires_ext_train_ridge with
 * opts; opts NULL = FP64 Gram, no washout): y[k] is T[k] x num_outputs_k, the
 * fitted W_out (num_outputs_k x N_k) is kept for spires_ext_batch_predict and
 * copied to w_out[k] when given. elapsed_ms: wall time of the call. */
spires_status spires_ext_batch_train_ridge(spires_ext_batch *b, const double *const *u,
                                           const double *const *y, const size_t *T,
                                           const double *lambda,
                                           const spires_ext_ridge_opts *opts,
                                           double *const *w_out, double *elapsed_ms);

/* Readouts y[k] (T[k] x num_outputs_k) of every instance over u[k] from reset
 * with its current W_out (same arithmetic as spires_run). */
spires_status spires_ext_batch_predict(spires_ext_batch *b, const double *const *u,
                                       const size_t *T, double *const *y,
                                       double *elapsed_ms);

/* Fit and score from one simulation: every instance runs T[k] steps of u[k]
 * from reset with its states recorded, its ridge readout is fitted on rows
 * [washout, T_fit[k]) against y[k] (T_fit[k] x num_outputs_k needed) and the
 * fitted W_out, kept for later calls and copied to w_out[k] when given, is
 * applied to all T[k] rows: y_out[k] is T[k] x num_outputs_k. */
spires_status spires_ext_batch_fit_predict(spires_ext_batch *b, const double *const *u,
                                           const double *const *y, const size_t *T,
                                           const size_t *T_fit, const double *lambda,
                                           const spires_ext_ridge_opts *opts,
                                           double *const *y_out, double *const *w_out,
                                           double *elapsed_ms);

/* Wall-clock milliseconds of spires_ext_batch_create: host construction of
 * the instances, and the device set-up (layouts, recurrent-input formats,
 * uploads). */
spires_status spires_ext_batch_timing(const spires_ext_batch *b, double *construct_ms,
                                      double *setup_ms);

/* Autotuner of the batched launch: runs the batch over u / T (lengths of a
 * representative sample, every instance from reset) once per candidate
 * schedule -- four families of CTA groups (size classes with power-of-two
 * widths, with exact minimum widths, with doubled widths; list scheduling
 * heaviest first) on a grid of full occupancy and on one CTA per SM -- and
 * keeps the one with the shortest device time for later runs. Returns the
 * chosen family (0..3), grid size and its time (any pointer may be NULL). */
spires_status spires_ext_batch_autotune(spires_ext_batch *b, const double *const *u,
                                        const size_t *T, int *schedule, int *ctas,
                                        double *best_ms);

/* Schedule of the last run: CTAs of the grid, CTA groups, and whether the
 * launch sequence runs as a CUDA graph (1) or as direct launches (-1). */
spires_status spires_ext_batch_info(const spires_ext_batch *b, int *ctas, int *groups,
                                    int *graph);

/* ---- surrogate network of the hyper-parameter search ----------------------
 * No counterpart in the reference. An MLP 10 -> 128 -> 128 -> 2 (GELU) that
 * predicts the mean and log-variance of a candidate's full-fidelity
 * log-NRMSE from 10 features (hyper-parameters and its low-fidelity loss),
 * trained on the GPU by hand-written forward, backward and Adam kernels on the
 * Gaussian negative log-likelihood 0.5 (v + (y - m)^2 exp(-v)) averaged over
 * the rows. FP32 parameters (layout: W1[128][10], b1[128], W2[128][128],
 * b2[128], W3[2][128], b3[2]); X is row-major n x 10; host arrays throughout. */
typedef struct spires_ext_mlp spires_ext_mlp;

size_t        spires_ext_mlp_num_params(void);
spires_status spires_ext_mlp_create(uint64_t seed, spires_ext_mlp **out);
void          spires_ext_mlp_destroy(spires_ext_mlp *m);
spires_status spires_ext_mlp_get_params(spires_ext_mlp *m, float *params);
/* also clears the Adam moments */
spires_status spires_ext_mlp_set_params(spires_ext_mlp *m, const float *params);
/* NLL over the n rows and its gradient (grad may be NULL); parameters unchanged */
spires_status spires_ext_mlp_loss_grad(spires_ext_mlp *m, const float *X, const float *y,
                                       size_t n, float *loss, float *grad);
/* Adam (beta 0.9 / 0.999, eps 1e-8) over `epochs` seeded shuffles in
 * minibatches of `batch` rows; final_loss = NLL of the last minibatch */
spires_status spires_ext_mlp_train(spires_ext_mlp *m, const float *X, const float *y, size_t n,
                                   int epochs, int batch, float lr, uint64_t seed,
                                   float *final_loss);
/* mean / logvar per row (either may be NULL); bf16 = 1: weights and
 * activations rounded to BF16, products and sums in FP32 on the CUDA cores
 * (the network is too small for the tensor cores to pay) */
spires_status spires_ext_mlp_predict(spires_ext_mlp *m, const float *X, size_t n, int bf16,
                                     float *mean, float *logvar);
long long     spires_ext_mlp_kernel_launches(const spires_ext_mlp *m);

#ifdef __cplusplus
}
#endif
#endif
