// pending.cu -- entry points whose kernels are being brought up; they report SLCS_ERR_INTERNAL.
#include "slcs_internal.cuh"

using namespace slcs;

extern "C" {
int slcs_scores(const int32_t *, int, int, const slcs_query *, int, int32_t *) {
    return fail(SLCS_ERR_INTERNAL, "score queries not available in this build");
}
int slcs_scores_dev(const int32_t *, int, int, const slcs_query *, int, int32_t *, void *) {
    return fail(SLCS_ERR_INTERNAL, "score queries not available in this build");
}
}
