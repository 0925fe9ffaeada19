// cmps::tf32_rna (integer rounding) against cvt.rna.tf32.f32, bit for bit,
// on 2^24 finite inputs: xorshift bit patterns, exact ties (bit 12 set, bits
// 0-11 clear) and subnormals.  Prints the mismatch count; exit status 0 when
// there is none.
#include <cstdint>
#include <cstdio>

#include "tf32_round.cuh"

__global__ void compare(const uint32_t* in, int n, unsigned long long* bad, uint32_t* first) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(__uint_as_float(in[i])));
  const uint32_t q = __float_as_uint(cmps::tf32_rna(__uint_as_float(in[i])));
  if (q != r && atomicAdd(bad, 1ull) == 0) {
    first[0] = in[i];
    first[1] = r;
    first[2] = q;
  }
}

int main() {
  const int n = 1 << 24;
  uint32_t* h = new uint32_t[n];
  uint64_t s = 88172645463325252ull;
  for (int i = 0; i < n; ++i) {
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    uint32_t u = (uint32_t)s;
    if ((u & 0x7F800000u) == 0x7F800000u) u &= 0xBFFFFFFFu;  // finite only
    if (i < 65536) u = (u & 0xFFFFE000u) | 0x1000u;        // exact ties
    else if (i < 131072) u &= 0x807FFFFFu;                 // subnormals
    h[i] = u;
  }
  uint32_t *d = nullptr, *first = nullptr;
  unsigned long long* bad = nullptr;
  if (cudaMalloc(&d, sizeof(uint32_t) * n) || cudaMalloc(&bad, 8) || cudaMalloc(&first, 12)) return 2;
  cudaMemset(bad, 0, 8);
  cudaMemset(first, 0, 12);
  cudaMemcpy(d, h, sizeof(uint32_t) * n, cudaMemcpyHostToDevice);
  compare<<<n / 256, 256>>>(d, n, bad, first);
  unsigned long long hb = 0;
  uint32_t hf[3] = {0, 0, 0};
  cudaMemcpy(&hb, bad, 8, cudaMemcpyDeviceToHost);
  cudaMemcpy(hf, first, 12, cudaMemcpyDeviceToHost);
  const cudaError_t e = cudaGetLastError();
  printf("cuda=%d mismatches=%llu of %d (first: in %08x cvt %08x int %08x)\n", (int)e, hb, n, hf[0], hf[1], hf[2]);
  cudaFree(d);
  cudaFree(bad);
  cudaFree(first);
  delete[] h;
  return (e != cudaSuccess || hb) ? 1 : 0;
}
