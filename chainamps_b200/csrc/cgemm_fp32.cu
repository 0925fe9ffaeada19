// Grouped complex GEMM in single precision (FP32 FFMA, FP32 accumulation):
// the low-precision form of the canonical-order H_eff matvec
// (canonical.cu).  Its stages contract one index of a few dozen states at a
// time (K = states per charge class, or an a-sector dimension), so they are
// bound by the bytes they move and by latency, not by a tensor pipe: halving
// the bytes per element (FP32 planes instead of FP64) is what the low
// precision buys here.
//
// Same work description as zgemm_grouped_fp64 (GemmTask / GemmTerm /
// GemmTile, K-concatenated terms, the two-level N index) and the same tile
// shapes (64 x 64, 32 x 128, 128 x 32), so one plan drives both precisions.
// 128 threads; thread (tm, tn) owns the 8 x 4 complex outputs (tm + i TM,
// tn + j TN): shared-memory reads and output stores run along consecutive
// threads.  Operands are staged global -> shared with 4-byte cp.async
// (zero-filled outside the block), double buffered; A is stored k-major in
// shared memory with one float of row padding (conflict-free transposing
// stores).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <string>

#include "internal.h"

namespace cmps {

namespace {

constexpr int BK = 16;
constexpr int NT = 128;
constexpr int RM = 8, RN = 4;  // complex outputs per thread: RM rows x RN columns

template <int BM, int BN>
struct Tile32 {
  static_assert((BM / RM) * (BN / RN) == NT, "one micro-tile per thread");
  static constexpr int TM = BM / RM, TN = BN / RN;
  static constexpr int LDA = BM + 1, LDB = BN;
  static constexpr int PLANE_A = BK * LDA, PLANE_B = BK * LDB;
  static constexpr int STAGE = 2 * PLANE_A + 2 * PLANE_B;  // floats: A re, A im, B re, B im
  static constexpr size_t SMEM_BYTES = 2 * (size_t)STAGE * sizeof(float);
};

__device__ __forceinline__ void cp_async4(float* smem, const float* gmem, bool pred) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int sz = pred ? 4 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }
__device__ __forceinline__ void cp_wait0() { asm volatile("cp.async.wait_group 0;\n" ::); }

template <bool NSPLIT>
__device__ __forceinline__ int64_t ncol(int n, int n_in, int ld_out) {
  if (!NSPLIT) return n;
  const int q = n / n_in;
  return (int64_t)q * ld_out + (n - q * n_in);
}

template <int BM, int BN, bool NSPLIT>
__device__ __forceinline__ void load_stage(float* buf, const GemmTerm& t, int k0, int m0, int n0, int M, int N,
                                           int n_in, const float* __restrict__ Ar, const float* __restrict__ Ai,
                                           const float* __restrict__ Br, const float* __restrict__ Bi) {
  using T = Tile32<BM, BN>;
  float* sAr = buf;
  float* sAi = buf + T::PLANE_A;
  float* sBr = buf + 2 * T::PLANE_A;
  float* sBi = sBr + T::PLANE_B;
  const int tid = threadIdx.x;
#pragma unroll
  for (int j = 0; j < (BM * BK) / NT; ++j) {
    const int idx = tid + j * NT;
    const int kk = idx % BK, mm = idx / BK;  // A[m][k]: consecutive threads along k
    const int gm = m0 + mm, gk = k0 + kk;
    const bool ok = gm < M && gk < t.k;
    const int64_t o = ok ? t.a_off + (int64_t)gm * t.lda + gk : 0;
    cp_async4(sAr + kk * T::LDA + mm, Ar + o, ok);
    cp_async4(sAi + kk * T::LDA + mm, Ai + o, ok);
  }
#pragma unroll
  for (int j = 0; j < (BN * BK) / NT; ++j) {
    const int idx = tid + j * NT;
    const int kk = idx / BN, nn = idx % BN;  // B[k][n]: along n
    const int gn = n0 + nn, gk = k0 + kk;
    const bool ok = gn < N && gk < t.k;
    const int64_t o = ok ? t.b_off + (int64_t)gk * t.ldb + ncol<NSPLIT>(gn, n_in, t.ldb_out) : 0;
    cp_async4(sBr + kk * T::LDB + nn, Br + o, ok);
    cp_async4(sBi + kk * T::LDB + nn, Bi + o, ok);
  }
}

template <int BM, int BN, bool NSPLIT>
__global__ void __launch_bounds__(NT, 3)
cgemm_grouped_fp32(const GemmTile* __restrict__ tiles, const GemmTask* __restrict__ tasks,
                   const GemmTerm* __restrict__ terms, const float* __restrict__ Ar, const float* __restrict__ Ai,
                   const float* __restrict__ Br, const float* __restrict__ Bi, float* __restrict__ Cr,
                   float* __restrict__ Ci) {
  using T = Tile32<BM, BN>;
  extern __shared__ float fsmem[];
  const GemmTile tile = tiles[blockIdx.x];
  const GemmTask task = tasks[tile.task];
  const int m0 = tile.m0, n0 = tile.n0, M = task.m, N = task.n;
  const int tm = threadIdx.x / T::TN, tn = threadIdx.x % T::TN;
  float accr[RM][RN], acci[RM][RN];
#pragma unroll
  for (int i = 0; i < RM; ++i)
#pragma unroll
    for (int j = 0; j < RN; ++j) accr[i][j] = acci[i][j] = 0.f;

  int cur_t = task.t0;
  int nxt_t = cur_t, nxt_k = 0;
  bool have = cur_t < task.t1;
  if (have) {
    const GemmTerm t = terms[cur_t];
    load_stage<BM, BN, NSPLIT>(fsmem, t, 0, m0, n0, M, N, task.n_in, Ar, Ai, Br, Bi);
    cp_commit();
    nxt_k = BK;
    if (nxt_k >= t.k) {
      nxt_t = cur_t + 1;
      nxt_k = 0;
    }
  }
  int stage = 0;
  while (have) {
    const bool more = nxt_t < task.t1;
    if (more) {
      const GemmTerm t = terms[nxt_t];
      load_stage<BM, BN, NSPLIT>(fsmem + (stage ^ 1) * T::STAGE, t, nxt_k, m0, n0, M, N, task.n_in, Ar, Ai, Br, Bi);
      cp_commit();
      cp_wait1();
    } else {
      cp_wait0();
    }
    __syncthreads();
    const float* sAr = fsmem + stage * T::STAGE;
    const float* sAi = sAr + T::PLANE_A;
    const float* sBr = sAr + 2 * T::PLANE_A;
    const float* sBi = sBr + T::PLANE_B;
#pragma unroll 4
    for (int kk = 0; kk < BK; ++kk) {
      float ar[RM], ai[RM], br[RN], bi[RN];
#pragma unroll
      for (int i = 0; i < RM; ++i) {
        ar[i] = sAr[kk * T::LDA + tm + i * T::TM];
        ai[i] = sAi[kk * T::LDA + tm + i * T::TM];
      }
#pragma unroll
      for (int j = 0; j < RN; ++j) {
        br[j] = sBr[kk * T::LDB + tn + j * T::TN];
        bi[j] = sBi[kk * T::LDB + tn + j * T::TN];
      }
#pragma unroll
      for (int i = 0; i < RM; ++i)
#pragma unroll
        for (int j = 0; j < RN; ++j) {
          accr[i][j] = fmaf(ar[i], br[j], accr[i][j]);
          accr[i][j] = fmaf(-ai[i], bi[j], accr[i][j]);
          acci[i][j] = fmaf(ar[i], bi[j], acci[i][j]);
          acci[i][j] = fmaf(ai[i], br[j], acci[i][j]);
        }
    }
    __syncthreads();
    have = more;
    if (more) {
      cur_t = nxt_t;
      const GemmTerm t = terms[cur_t];
      nxt_k += BK;
      if (nxt_k >= t.k) {
        nxt_t = cur_t + 1;
        nxt_k = 0;
      }
      stage ^= 1;
    }
  }
#pragma unroll
  for (int i = 0; i < RM; ++i)
#pragma unroll
    for (int j = 0; j < RN; ++j) {
      const int gm = m0 + tm + i * T::TM, gn = n0 + tn + j * T::TN;
      if (gm < M && gn < N) {
        const int64_t o = task.c_off + (int64_t)gm * task.ldc + ncol<NSPLIT>(gn, task.n_in, task.ldc_out);
        Cr[o] = accr[i][j];
        Ci[o] = acci[i][j];
      }
    }
}

template <int BM, int BN, bool NSPLIT>
int launch32(const GemmPlan& p, const Planar32& A, const Planar32& B, Planar32& C, cudaStream_t st) {
  using T = Tile32<BM, BN>;
  CMPS_TRY(ensure_smem_optin((const void*)cgemm_grouped_fp32<BM, BN, NSPLIT>, (int)T::SMEM_BYTES));
  if (p.tiles.empty()) return CMPS_OK;
  const int64_t ntiles = (int64_t)p.tiles.size();
  if (ntiles > 0x7fffffff) return fail(CMPS_ERR_ARG, "too many GEMM tiles");
  cgemm_grouped_fp32<BM, BN, NSPLIT><<<(unsigned)ntiles, NT, T::SMEM_BYTES, st>>>(
      p.d_tiles, p.d_tasks, p.d_terms, A.re(), A.im(), B.re(), B.im(), C.re(), C.im());
  CMPS_CUDA(cudaGetLastError());
  return CMPS_OK;
}

template <int BM, int BN>
int launch32_shape(const GemmPlan& p, const Planar32& A, const Planar32& B, Planar32& C, cudaStream_t st) {
  return p.nsplit ? launch32<BM, BN, true>(p, A, B, C, st) : launch32<BM, BN, false>(p, A, B, C, st);
}

__global__ void k_to_f32(const double* __restrict__ re, const double* __restrict__ im, int64_t n,
                         float* __restrict__ ore, float* __restrict__ oim) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    ore[e] = (float)re[e];
    oim[e] = (float)im[e];
  }
}
__global__ void k_to_f64(const float* __restrict__ re, const float* __restrict__ im, int64_t n,
                         double* __restrict__ ore, double* __restrict__ oim) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    ore[e] = (double)re[e];
    oim[e] = (double)im[e];
  }
}

unsigned grid_for(int64_t n) { return (unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16); }

}  // namespace

int Planar32::alloc(int64_t n) {
  release();
  len = n;
  if (dmalloc(&d, sizeof(float) * 2 * std::max<int64_t>(n, 1)) != cudaSuccess) {
    d = nullptr;
    len = 0;
    return fail(CMPS_ERR_NOMEM, "device allocation failed (" + std::to_string(8 * n) + " bytes)");
  }
  owned = true;
  return CMPS_OK;
}

void Planar32::release() {
  if (d && owned) dfree(d);
  d = nullptr;
  len = 0;
  owned = false;
}

int launch_cgemm_fp32(const GemmPlan& p, const Planar32& A, const Planar32& B, Planar32& C, cudaStream_t st) {
  switch (p.shape) {
    case 0: return launch32_shape<64, 64>(p, A, B, C, st);
    case 1: return launch32_shape<32, 128>(p, A, B, C, st);
    case 2: return launch32_shape<128, 32>(p, A, B, C, st);
    default: return fail(CMPS_ERR_STATE, "GEMM plan not uploaded (no tile shape)");
  }
}

int to_fp32(const double* re, const double* im, int64_t n, Planar32& out, cudaStream_t st) {
  if (n > out.len) return fail(CMPS_ERR_STATE, "FP32 conversion: destination too short");
  if (n == 0) return CMPS_OK;
  k_to_f32<<<grid_for(n), 256, 0, st>>>(re, im, n, out.re(), out.im());
  CMPS_CUDA(cudaGetLastError());
  return CMPS_OK;
}

int to_fp64(const Planar32& in, int64_t n, double* re, double* im, cudaStream_t st) {
  if (n > in.len) return fail(CMPS_ERR_STATE, "FP64 conversion: source too short");
  if (n == 0) return CMPS_OK;
  k_to_f64<<<grid_for(n), 256, 0, st>>>(in.re(), in.im(), n, re, im);
  CMPS_CUDA(cudaGetLastError());
  return CMPS_OK;
}

}  // namespace cmps
