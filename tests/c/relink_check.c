/*
 * relink_check.c -- a C caller of the spires API, built against a spires.h
 * and linked against this library's libspires.so. It names every function of
 * the API with its declared type (so the compiler checks each signature) and
 * calls the ones that need no GPU with invalid arguments, checking the status
 * codes. Built by tests/test_c_abi.py against include/spires.h and, when it is
 * available, against the original project's header.
 */
#include <stdio.h>
#include <stdlib.h>
#include "spires.h"

#define CHECK(cond)                                                    \
    do {                                                               \
        if (!(cond)) {                                                 \
            fprintf(stderr, "check failed: %s (line %d)\n", #cond, __LINE__); \
            return 1;                                                  \
        }                                                              \
    } while (0)

int main(void)
{
    /* every entry point with the type the header declares */
    spires_status (*p_create)(const spires_reservoir_config *, spires_reservoir **) =
        spires_reservoir_create;
    void (*p_destroy)(spires_reservoir *) = spires_reservoir_destroy;
    spires_status (*p_reset)(spires_reservoir *) = spires_reservoir_reset;
    spires_status (*p_step)(spires_reservoir *, const double *) = spires_step;
    double *(*p_run)(spires_reservoir *, const double *, size_t) = spires_run;
    spires_status (*p_online)(spires_reservoir *, const double *, double) = spires_train_online;
    spires_status (*p_ridge)(spires_reservoir *, const double *, const double *, size_t,
                             double) = spires_train_ridge;
    spires_status (*p_rls)(spires_reservoir *, const double *, const double *, size_t, double,
                           double) = spires_train_rls;
    spires_status (*p_coarse)(const spires_reservoir *, double, spires_reservoir **) =
        spires_coarse_grain;
    double *(*p_copy_state)(spires_reservoir *) = spires_copy_reservoir_state;
    spires_status (*p_read_state)(spires_reservoir *, double *) = spires_read_reservoir_state;
    spires_status (*p_read_spikes)(spires_reservoir *, double *) = spires_read_spike_state;
    double *(*p_copy_w)(const spires_reservoir *) = spires_copy_weights;
    spires_status (*p_read_w)(const spires_reservoir *, double *) = spires_read_weights;
    spires_status (*p_out)(spires_reservoir *, double *) = spires_compute_output;
    double *(*p_copy_ro)(const spires_reservoir *) = spires_copy_readout;
    spires_status (*p_read_ro)(const spires_reservoir *, double *) = spires_read_readout;
    size_t (*p_nn)(const spires_reservoir *) = spires_num_neurons;
    size_t (*p_ni)(const spires_reservoir *) = spires_num_inputs;
    size_t (*p_no)(const spires_reservoir *) = spires_num_outputs;
    int (*p_opt)(const spires_reservoir_config *, const struct spires_opt_budget *, int,
                 const struct spires_opt_score *, struct spires_opt_result *, const double *,
                 const double *, size_t) = spires_optimize;
    void *all[] = {(void *)p_create, (void *)p_destroy, (void *)p_reset, (void *)p_step,
                   (void *)p_run, (void *)p_online, (void *)p_ridge, (void *)p_rls,
                   (void *)p_coarse, (void *)p_copy_state, (void *)p_read_state,
                   (void *)p_read_spikes, (void *)p_copy_w, (void *)p_read_w, (void *)p_out,
                   (void *)p_copy_ro, (void *)p_read_ro, (void *)p_nn, (void *)p_ni,
                   (void *)p_no, (void *)p_opt};
    for (size_t k = 0; k < sizeof(all) / sizeof(all[0]); ++k)
        CHECK(all[k] != NULL);

    /* enumerator values and layout the callers compile in */
    CHECK(SPIRES_OK == 0 && SPIRES_ERR_INVALID_ARG == 1 && SPIRES_ERR_ALLOC == 2 &&
          SPIRES_ERR_INTERNAL == 3);
    CHECK(SPIRES_NEURON_FLIF_GL == 3 && SPIRES_SYNAPSE_FRACTIONAL_MULTIEXP == 4);
    CHECK(SPIRES_CONN_SCALE_FREE == 2);

    /* calls that need no GPU: argument checks */
    spires_reservoir *r = NULL;
    CHECK(spires_reservoir_create(NULL, &r) == SPIRES_ERR_INVALID_ARG);
    spires_reservoir_destroy(NULL);
    CHECK(spires_reservoir_reset(NULL) == SPIRES_ERR_INVALID_ARG);
    CHECK(spires_step(NULL, NULL) == SPIRES_ERR_INVALID_ARG);
    CHECK(spires_run(NULL, NULL, 0) == NULL);
    CHECK(spires_read_reservoir_state(NULL, NULL) == SPIRES_ERR_INVALID_ARG);
    CHECK(spires_num_neurons(NULL) == 0 && spires_num_inputs(NULL) == 0 &&
          spires_num_outputs(NULL) == 0);
    spires_reservoir_config bad = {0};
    bad.dt = 0.3; /* 1/dt is not an integer */
    CHECK(spires_reservoir_create(&bad, &r) == SPIRES_ERR_INVALID_ARG);
    printf("relink check ok\n");
    return 0;
}
