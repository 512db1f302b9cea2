/*
 * coarse.c -- spires_coarse_grain (src/reservoir.c:782-967, src/spires_api.c:226-245).
 *
 * Pair-merging of neurons joined by a strong weight, repeated until a full
 * pass merges nothing, then a new reservoir over the survivors. The merge
 * loop runs on the device (dev_coarse.cu, bit-identical to the reference's
 * loop); the dense matrices are assembled and compacted here and the new
 * reservoir gets its own device state. As in the reference
 * the merged matrix is installed without a spectral rescale and without new
 * W_in/W_out draws (PSC_HETEROGENEOUS still draws per-edge tau for it).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "../../include/spires.h"
#include "sp_model.h"
#include "sp_dev.h"
#include "sp_api_internal.h"

#define SPIRES_EXPORT __attribute__((visibility("default")))

SPIRES_EXPORT spires_status spires_coarse_grain(const spires_reservoir *r, double weight_threshold,
                                                spires_reservoir **out_r)
{
    if (!r || !r->dev || !out_r)
        return SPIRES_ERR_INVALID_ARG;
    /* Below zero (or NaN) every pass merges again -- the zeroed rows of merged
     * neurons pass the test -- and the reference's loop never ends; refuse
     * such thresholds instead. */
    if (!(weight_threshold >= 0.0))
        return SPIRES_ERR_INVALID_ARG;
    const sp_host_model *m = &r->m;
    const size_t n = m->n, nin = m->din, nout = m->dout;
    spires_status st = SPIRES_ERR_ALLOC;

    double *W = calloc(n * n, sizeof(double));
    double *Win = malloc(((n) * (nin) > 0 ? (n) * (nin) : 1) * sizeof(double));
    double *Wout = malloc(((n) * (nout) > 0 ? (n) * (nout) : 1) * sizeof(double));
    double *V = malloc(n * sizeof(double));
    int *alive = malloc(n * sizeof(int));
    size_t *old_to_new = malloc(n * sizeof(size_t));
    double *Wn = NULL, *Winn = NULL, *Woutn = NULL;
    sp_host_model nm;
    memset(&nm, 0, sizeof(nm));
    if (!W || !Win || !Wout || !V || !alive || !old_to_new)
        goto done;

    for (size_t i = 0; i < n; i++)
        for (int64_t k = m->row_ptr[i]; k < m->row_ptr[i + 1]; k++)
            W[i * n + (size_t)m->col[k]] = m->w[k];
    memcpy(Win, m->W_in, n * nin * sizeof(double));
    memcpy(Wout, m->W_out, n * nout * sizeof(double));
    if (sp_dev_read_state(r->dev, V) != SP_OK) {
        st = SPIRES_ERR_INTERNAL;
        goto done;
    }
    for (size_t i = 0; i < n; i++)
        alive[i] = 1;

    /* the merge loop (src/reservoir.c:822-915) runs on the device */
    {
        int rc0 = sp_coarse_merge_device(n, nin, nout, weight_threshold, W, Win, Wout, V, alive);
        if (rc0) {
            st = (rc0 == SP_EALLOC) ? SPIRES_ERR_ALLOC : SPIRES_ERR_INTERNAL;
            goto done;
        }
    }

    size_t ns = 0;
    for (size_t i = 0; i < n; i++)
        old_to_new[i] = alive[i] ? ns++ : (size_t)-1;
    Wn = calloc(ns * ns > 0 ? ns * ns : 1, sizeof(double));
    Winn = calloc(ns * nin > 0 ? ns * nin : 1, sizeof(double));
    Woutn = calloc(ns * nout > 0 ? ns * nout : 1, sizeof(double));
    if (!Wn || !Winn || !Woutn)
        goto done;
    for (size_t i = 0; i < n; i++) {
        if (!alive[i])
            continue;
        size_t a = old_to_new[i];
        for (size_t j = 0; j < n; j++)
            if (alive[j])
                Wn[a * ns + old_to_new[j]] = W[i * n + j];
        for (size_t k = 0; k < nin; k++)
            Winn[a * nin + k] = Win[i * nin + k];
        for (size_t o = 0; o < nout; o++)
            Woutn[o * ns + a] = Wout[o * n + i];
    }

    /* new model: same configuration, merged weights */
    nm.n = ns;
    nm.din = nin;
    nm.dout = nout;
    nm.spectral_radius = m->spectral_radius;
    nm.ei_ratio = m->ei_ratio;
    nm.input_strength = m->input_strength;
    nm.connectivity = m->connectivity;
    nm.dt = m->dt;
    nm.conn_type = m->conn_type;
    nm.neuron_type = m->neuron_type;
    nm.syn_type = m->syn_type;
    nm.syn_backend = m->syn_backend;
    nm.neuron_params = m->neuron_params;
    nm.synapse_params = m->synapse_params;
    nm.micro_steps = m->micro_steps;
    nm.diffusive_seed = m->diffusive_seed;
    int rc = sp_model_derive_neuron(&nm);
    if (!rc)
        rc = sp_model_set_dense_weights(&nm, Wn);
    if (rc) {
        st = (rc == SP_EALLOC) ? SPIRES_ERR_ALLOC : SPIRES_ERR_INTERNAL;
        goto done;
    }
    nm.W_in = Winn;
    nm.W_out = Woutn;
    Winn = Woutn = NULL;

    spires_reservoir *nr = NULL;
    rc = sp_handle_from_model(&nm, &nr);
    if (rc) {
        st = (rc == SP_EALLOC) ? SPIRES_ERR_ALLOC : SPIRES_ERR_INTERNAL;
        goto done;
    }
    /* set_neuron_state: membrane potential only (src/reservoir.c:956-962) */
    {
        size_t idx = 0;
        for (size_t i = 0; i < n; i++)
            if (alive[i])
                V[idx++] = V[i];
        if (sp_dev_set_state(nr->dev, V) != SP_OK) {
            spires_reservoir_destroy(nr);
            st = SPIRES_ERR_INTERNAL;
            goto done;
        }
    }
    *out_r = nr;
    st = SPIRES_OK;
done:
    sp_model_free(&nm);
    free(W);
    free(Win);
    free(Wout);
    free(V);
    free(alive);
    free(old_to_new);
    free(Wn);
    free(Winn);
    free(Woutn);
    return st;
}
