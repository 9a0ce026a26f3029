// Placeholder entry points for solvers not built yet.
#include "amk_internal.cuh"

namespace amk {

int fmm_forces(amk_ctx*, const View&, int, double, long, bool, double*) {
  return fail(AMK_ERR_UNSUPPORTED, "FMM solver not built");
}

}  // namespace amk

void fmm_destroy(amk_ctx*) {}
void mlp_destroy(amk_ctx*) {}
