// Entry points of parts not built yet.
#include "amk_internal.cuh"

void mlp_destroy(amk_ctx*) {}
