// Entry points declared in lamb_gpu.h whose implementation is not built yet:
// they return lamb_unimplemented (src/lamb_error.F90:157).
#include "common.cuh"

using namespace lamb;

#define LAMB_PENDING(ctxp) \
  return fail(reinterpret_cast<Ctx*>(ctxp), LAMB_LEVEL_FAILURE, LAMB_TYPE_UNIMPLEMENTED, "not built yet")

extern "C" {
int32_t lamb_gpu_batch_create(lamb_gpu_ctx* c, const lamb_gpu_matrix*, const lamb_gpu_matrix*, const lamb_gpu_matrix*,
                              int32_t, double, lamb_gpu_batch**) { LAMB_PENDING(c); }
int32_t lamb_gpu_batch_execute(lamb_gpu_batch*, lamb_gpu_mult_stats*) {
  return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_UNIMPLEMENTED);
}
int32_t lamb_gpu_batch_destroy(lamb_gpu_batch*) { return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_UNIMPLEMENTED); }
}
