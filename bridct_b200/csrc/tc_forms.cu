// Tensor-core precision forms (placeholder until the tcgen05 kernels land).
#include "../../include/bridct_b200.h"
#include "bridct_internal.h"

namespace bridct {
int apply_tc_form(bridct_plan* p, int mode, int form, const float* x, float* y, size_t batch,
                  void* stream) {
  (void)p; (void)mode; (void)x; (void)y; (void)batch; (void)stream;
  set_error("tensor-core form " + std::to_string(form) + " is not available in this build");
  return BRIDCT_INVALID_ARGUMENT;
}
}  // namespace bridct
