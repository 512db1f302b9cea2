/*
 * sp_dev.h -- C ABI of the CUDA layer (device state of one reservoir).
 *
 * The host C code (api.c) owns an sp_host_model and one sp_dev per reservoir.
 * Every function returns an SP_* status; CUDA errors map to SP_EINTERNAL and
 * device allocation failures to SP_EALLOC. No function allocates device memory
 * except sp_dev_create, sp_dev_destroy-paired buffers and the ridge/RLS
 * working sets (which the reference also allocates per call).
 */
#ifndef SP_DEV_H
#define SP_DEV_H

#include <stddef.h>
#include <stdint.h>
#include "sp_model.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sp_dev sp_dev;

/* Launch shape of the persistent step kernel. */
typedef struct {
    int ctas;        /* CTAs in the cooperative grid (1 = no grid barrier) */
    int warps_max;   /* warps per CTA (blockDim = 32 * warps_max) */
    int variant;     /* 0 = generic ring loads, 1 = bulk-copy ring pipeline (FLIF_GL) */
    int stages;      /* pipeline depth of variant 1 */
    int rows;        /* ring rows per stage of variant 1 */
    int csr_global;  /* 1: SIMPLE synapse rows walked in global memory even when
                        the CTA's CSR slice fits in shared memory */
    int l2_pin;      /* variant 1: the oldest l2_pin lags of a step read with L2
                        evict-last priority, younger lags and ring writes
                        evict-first; 0 = no cache hints, -1 = automatic
                        (sp_dev_l2_pin_rows) */
} sp_launch;

int  sp_dev_create(const sp_host_model *m, sp_dev **out);
void sp_dev_destroy(sp_dev *d);

/* Re-initialise neuron state from m->nc (spike flags cleared, ring refilled,
 * internal step = 0). Synapse state is left as it is, as in the reference. */
int  sp_dev_reset_neurons(sp_dev *d, const sp_host_model *m);

/* Run T macro steps. `u` holds T x din inputs; `u_on_device` says whether it is
 * a device pointer (else host, staged in chunks); u == NULL means zeros.
 * Optional device outputs: phi [T x n] states after each macro step, raster
 * [T x nwords] spike words after each macro step, y [T x dout] readouts.
 * Host outputs (h_*) are filled chunk by chunk when the device ones are NULL. */
typedef struct {
    const double *u;
    int u_on_device;
    size_t T;
    double *d_phi;
    uint32_t *d_raster;
    double *d_y;
    double *h_phi;
    uint32_t *h_raster;
    double *h_y;
    int sync;        /* wait for completion and report kernel errors */
} sp_run_args;

int  sp_dev_run(sp_dev *d, const sp_run_args *a);
int  sp_dev_sync(sp_dev *d);

int  sp_dev_read_state(sp_dev *d, double *h_V);
int  sp_dev_read_spikes(sp_dev *d, double *h_spk);
int  sp_dev_set_state(sp_dev *d, const double *h_V);
int  sp_dev_compute_output(sp_dev *d, double *h_y);
int  sp_dev_upload_w_out(sp_dev *d, const double *h_W_out);
int  sp_dev_download_w_out(sp_dev *d, double *h_W_out);
void *sp_dev_stream(sp_dev *d);
int  sp_dev_get_launch(sp_dev *d, sp_launch *l);
/* Ring lags the launch keeps L2-resident (its l2_pin with -1 resolved). */
int  sp_dev_l2_pin_rows(const sp_dev *d);
int  sp_dev_set_launch(sp_dev *d, const sp_launch *l);
int  sp_dev_set_seed(sp_dev *d, uint64_t seed);
int  sp_dev_autotune(sp_dev *d, size_t steps);
/* State checkpoint: every mutable buffer of the dynamics and the step
 * counters, to and from a host buffer of sp_dev_state_bytes bytes. */
size_t sp_dev_state_bytes(sp_dev *d);
int  sp_dev_state_save(sp_dev *d, void *buf);
int  sp_dev_state_load(sp_dev *d, const void *buf);
/* Bounded waits of the step kernel: their limit in milliseconds (default
 * 2000); a one-shot hook that makes CTA `cta` withhold its grid-barrier
 * arrival at micro-step `micro_step` of the next launch (counted from that
 * launch's start), so that every other CTA's wait runs out; the code and
 * micro-step of the last device error the host read. */
int  sp_dev_set_wait_limit(sp_dev *d, double ms);
int  sp_dev_hold_arrival(sp_dev *d, int cta, long long micro_step);
int  sp_dev_last_error(const sp_dev *d, int *code, long long *micro_step);
/* SP_OK when buf's header matches this reservoir's sizes; touches nothing */
int  sp_dev_state_check(sp_dev *d, const void *buf);
size_t sp_dev_nwords(const sp_dev *d);
long long sp_dev_kernel_launches(const sp_dev *d);

/* Merge loop of spires_coarse_grain on the device (dev_coarse.cu), in place
 * on host arrays W [n][n], Win [n][nin], Wout [nout][n], V [n], alive [n]. */
int sp_coarse_merge_device(size_t n, size_t nin, size_t nout, double thr, double *W,
                           double *Win, double *Wout, double *V, int *alive);

/* Readouts on the device (dev_readout.cu). */
typedef struct {
    int gram_mode;      /* SP_GRAM_*: 0 FP64 Gram, 1 BF16X3, 2 TF32X3, 3 INT8 slices */
    int max_refine;     /* iterative-refinement sweeps */
    double refine_tol;  /* stop when ||r|| / ||b|| falls below */
    size_t washout;     /* rows of phi skipped before the Gram */
    int gram_slices;    /* INT8 mode: integer slices (2..8), 0 = default (7) */
} sp_ridge_opts;

typedef struct {
    int gram_mode_used;
    int refine_iters;
    double rel_residual;      /* ||B - (G + lambda I) W|| / ||B|| in FP64 */
    double gram_ms, factor_ms, refine_ms, collect_ms;
    int factor_failed;        /* Cholesky met a non-positive pivot */
    int lu_fallback;          /* solved by pivoted LU instead */
    int dual;                 /* solved in the dual form (fewer rows than n / 2) */
    double solve_ms;          /* first triangular solve (factor_ms: the factorisation) */
} sp_ridge_report;

int sp_dev_train_ridge(sp_dev *d, const sp_host_model *m, const double *h_u,
                       const double *h_y, size_t T, double lambda,
                       const sp_ridge_opts *o, sp_ridge_report *rep,
                       double *h_W_out);
int sp_ridge_host(const double *h_phi, size_t T, int n, const double *h_y, int dout,
                  double lambda, const sp_ridge_opts *o, sp_ridge_report *rep,
                  double *h_w_out);
int sp_dev_train_rls(sp_dev *d, const sp_host_model *m, const double *h_u,
                     const double *h_y, size_t T, double delta, double lambda,
                     double *h_W_out);
int sp_dev_train_online(sp_dev *d, const double *h_target, double lr,
                        double *h_W_out);

/* Surrogate MLP 10 -> 128 -> 128 -> 2 (dev_surrogate.cu). */
typedef struct sp_mlp sp_mlp;
int  sp_mlp_num_params(void);
int  sp_mlp_create(uint64_t seed, sp_mlp **out);
void sp_mlp_destroy(sp_mlp *m);
int  sp_mlp_get_params(sp_mlp *m, float *h);
int  sp_mlp_set_params(sp_mlp *m, const float *h);
int  sp_mlp_loss_grad(sp_mlp *m, const float *X, const float *y, int n, float *loss,
                      float *grad);
int  sp_mlp_train(sp_mlp *m, const float *X, const float *y, int n, int epochs, int batch,
                  float lr, uint64_t seed, float *final_loss);
int  sp_mlp_predict(sp_mlp *m, const float *X, int n, int bf16, float *mean, float *logvar);
long long sp_mlp_launches(const sp_mlp *m);

/* Current CUDA device of the calling thread (-1 = none) and selection of it
 * on a worker thread. */
int  sp_dev_current_device(void);
void sp_dev_use_device(int d);

/* Batched multi-reservoir path (dev_batch.cu): LIF_DISCRETE / FLIF_GL with
 * SIMPLE synapses. sp_batch_create takes over the models' buffers (the array
 * is zeroed). Every run starts all instances from their reset state. */
typedef struct sp_batch sp_batch;
int  sp_batch_create(sp_host_model *models, size_t count, sp_batch **out);
void sp_batch_destroy(sp_batch *b);
int  sp_batch_run(sp_batch *b, const double *const *u, const size_t *T,
                  uint32_t *const *raster, double *const *final_state, double *elapsed_ms);
int  sp_batch_train_ridge(sp_batch *b, const double *const *u, const double *const *y,
                          const size_t *T, const double *lambda, const sp_ridge_opts *o,
                          double *const *w_out, double *elapsed_ms);
int  sp_batch_predict(sp_batch *b, const double *const *u, const size_t *T,
                      double *const *y, double *elapsed_ms);
int  sp_batch_fit_predict(sp_batch *b, const double *const *u, const double *const *y,
                          const size_t *T, const size_t *T_fit, const double *lambda,
                          const sp_ridge_opts *o, double *const *y_out, double *const *w_out,
                          double *elapsed_ms);
int  sp_batch_info(const sp_batch *b, int *ctas, int *groups, int *graph);
int  sp_batch_autotune(sp_batch *b, const double *const *u, const size_t *T, int *best_mode,
                       int *best_ctas, double *best_ms);

#ifdef __cplusplus
}
#endif
#endif
