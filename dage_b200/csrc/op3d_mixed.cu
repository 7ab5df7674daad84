// op3d_mixed.cu -- split-precision tensor-core path (placeholder until the
// tcgen05 kernel lands): every entry point reports the path as unsupported.
#include "op3d.cuh"

namespace dage {
int mixed_setup(dage_op3d *) { return fail(DAGE_E_UNSUPPORTED, "mixed precision not built"); }
int mixed_apply(dage_op3d *, const double *, double *, cudaStream_t) {
  return fail(DAGE_E_UNSUPPORTED, "mixed precision not built");
}
int mixed_set_weights(dage_op3d *) { return 0; }
void mixed_destroy(dage_op3d *) {}
}  // namespace dage
