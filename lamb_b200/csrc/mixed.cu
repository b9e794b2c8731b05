// Mixed-precision numeric phase (int8 split slices on the tensor cores).
#include "multiply.cuh"

namespace lamb {

int32_t numeric_mixed(Ctx* ctx, DevMatrix*, DevMatrix*, DevMatrix*, const Symbolic&, const Work*, const int32_t*,
                      double*, int* slices_used) {
  *slices_used = 0;
  return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_UNIMPLEMENTED, "mixed precision not built yet");
}

}  // namespace lamb
