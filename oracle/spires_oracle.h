/*
 * oracle/spires_oracle.h -- TEST INFRASTRUCTURE ONLY: CPU restatement of the
 * reference reservoir dynamics and readouts, used as the checker for the GPU
 * library. Never linked into the product.
 *
 * Parity is pinned: tests/test_oracle.py checks this restatement bit for bit
 * against the reference sources compiled unchanged (oracle/_ref) and against
 * the committed fixtures in tests/golden/.
 */
#ifndef SPIRES_ORACLE_H
#define SPIRES_ORACLE_H

#include <stddef.h>
#include <stdint.h>

typedef struct {
    int neuron_type;          /* 0..4 as spires_neuron_type */
    int synapse_type;         /* 0..4 as spires_synapse_type */
    int n, din, dout;
    double dt, input_strength;
    const double *neuron_params;
    const double *synapse_params;
    const int64_t *row_ptr;   /* CSR of W, ascending columns */
    const int32_t *col;
    const double *val;
    const double *w_in;       /* n x din */
    const double *w_out;      /* dout x n */
    const double *edge_tau;   /* PSC_HETEROGENEOUS: tau per CSR edge */
    uint64_t diffusive_seed;  /* FLIF_DIFFUSIVE stream seed (alpha < 1 only) */
} orc_model;

typedef struct orc_state orc_state;

orc_state *orc_create(const orc_model *m);
void orc_free(orc_state *s);
void orc_reset(orc_state *s);                 /* neurons only (src/reservoir.c:770-780) */
void orc_step(orc_state *s, const double *u); /* one macro step; u may be NULL */
void orc_state_read(const orc_state *s, double *V, double *spikes);
void orc_output(const orc_state *s, double *y);
/* T macro steps; phi [T x n] and raster [T x n] (0/1 bytes) optional */
void orc_run(orc_state *s, const double *u, size_t T, double *phi, uint8_t *raster, double *y);

/* FP64 ridge on a recorded state matrix: W_out = (X^T X + lam I)^-1 X^T Y,
 * rows [washout, T) of X (T x n) and Y (T x dout); LU with partial pivoting.
 * Returns 0 on success. */
int orc_ridge(const double *X, const double *Y, size_t T, size_t washout, int n, int dout,
              double lam, double *w_out /* dout x n */);

/* readout training restated from src/reservoir.c: w_out (dout x n) in/out */
void orc_train_online(orc_state *s, const double *target, double lr, double *w_out);
int  orc_train_rls(orc_state *s, const double *u, const double *y, size_t T, double delta,
                   double lambda, double *w_out);

#endif
