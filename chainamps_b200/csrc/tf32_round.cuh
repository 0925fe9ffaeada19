// TF32 rounding used by the split-precision converter warps.
#pragma once

#include <stdint.h>

namespace cmps {

// x rounded to TF32 (10 explicit mantissa bits), to nearest with ties away
// from zero, for finite x: half a TF32 unit (bit 12) is added to the
// magnitude bits and the 13 low bits are cleared; a mantissa carry moves into
// the exponent, which is the correctly rounded result.  Two integer
// operations at full rate, where a conversion instruction runs at a fraction
// of it (the converter warps round 64 values per row and k-step).  Equal bit
// for bit to cvt.rna.tf32.f32 on finite inputs (tests/cuda/tf32_round_check.cu).
__device__ __forceinline__ float tf32_rna(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

}  // namespace cmps
