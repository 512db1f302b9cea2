// gram_tc.cu -- placeholder until the tcgen05 BF16x3 Gram lands.
#include "sp_gram.h"
#include "sp_model.h"
extern "C" int sp_gram_bf16x3_available(void) { return 0; }
extern "C" int sp_gram_bf16x3(cudaStream_t, const double *, int, size_t, size_t, double *, int)
{
    return SP_EINTERNAL;
}
