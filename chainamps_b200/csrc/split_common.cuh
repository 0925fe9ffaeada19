// Splitting FP64 complex operands into the planes of the tcgen05 split
// forms (internal; shared by the folded and the canonical split operators).
//  * TF32: re_hi, re_lo, im_hi, im_lo with hi = x rounded to TF32 (round to
//    nearest, ties away) and lo = x - hi rounded to TF32;
//  * BF16: re_hi, re_mid, im_hi, im_mid with hi = x rounded to BF16 and
//    mid = x - hi rounded to BF16, stored as raw 16-bit patterns.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace cmps {
namespace {

__device__ __forceinline__ float rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}
__device__ __forceinline__ void split4(double re, double im, float* p0, float* p1, float* p2, float* p3) {
  const float hr = rna((float)re), hi = rna((float)im);
  *p0 = hr;
  *p1 = rna((float)(re - (double)hr));
  *p2 = hi;
  *p3 = rna((float)(im - (double)hi));
}
// BF16: hi = x rounded to BF16, mid = x - hi rounded to BF16 (raw bits)
__device__ __forceinline__ void split4(double re, double im, uint16_t* p0, uint16_t* p1, uint16_t* p2,
                                       uint16_t* p3) {
  const __nv_bfloat16 hr = __double2bfloat16(re), hi = __double2bfloat16(im);
  *p0 = __bfloat16_as_ushort(hr);
  *p1 = __bfloat16_as_ushort(__double2bfloat16(re - (double)__bfloat162float(hr)));
  *p2 = __bfloat16_as_ushort(hi);
  *p3 = __bfloat16_as_ushort(__double2bfloat16(im - (double)__bfloat162float(hi)));
}

struct SplitBlock {
  int64_t src_off, dst_off;
  int32_t rows, cols, ld_dst, transpose;
};

// dst (4 planes) <- split(src block), optionally transposed.
template <class E>
__global__ void k_split_blocks(const SplitBlock* __restrict__ blocks, const double* __restrict__ sr,
                               const double* __restrict__ si, E* __restrict__ dst, int64_t plane) {
  const SplitBlock b = blocks[blockIdx.x];
  const int64_t n = (int64_t)b.rows * b.cols;
  for (int64_t e = threadIdx.x; e < n; e += blockDim.x) {
    const int64_t r = e / b.cols, c = e % b.cols;
    const int64_t o = b.transpose ? b.dst_off + c * b.ld_dst + r : b.dst_off + r * b.ld_dst + c;
    split4(sr[b.src_off + e], si[b.src_off + e], dst + o, dst + o + plane, dst + o + 2 * plane, dst + o + 3 * plane);
  }
}

}  // namespace
}  // namespace cmps
