// Split-precision (3-term TF32 on tcgen05, FP32 accumulate) operand
// preparation.  The FP64 path needs nothing extra.
#include "heff.h"

namespace cmps {

int prepare_precision(Heff* h, int precision) {
  if (precision == CMPS_FP64) return CMPS_OK;
  (void)h;
  return fail(CMPS_ERR_ARG, "split-TF32 contraction path is not available in this build");
}

}  // namespace cmps
