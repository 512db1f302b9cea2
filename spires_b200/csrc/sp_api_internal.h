/*
 * sp_api_internal.h -- the opaque handle behind spires_reservoir and helpers
 * shared by the host C files (api.c, coarse.c, optimize.c).
 */
#ifndef SP_API_INTERNAL_H
#define SP_API_INTERNAL_H

#include "sp_model.h"
#include "sp_dev.h"

struct spires_reservoir {
    sp_host_model m;  /* configuration, weights (host copy), constants */
    sp_dev *dev;      /* device state */
};

/* Gram precision used by spires_train_ridge: FP64 unless the environment
 * variable SPIRES_RIDGE_GRAM selects "bf16x3". */
int sp_default_gram_mode(void);

/* Wrap a built host model into a handle (moves ownership of the model). */
int sp_handle_from_model(sp_host_model *m, struct spires_reservoir **out_r);

#endif
