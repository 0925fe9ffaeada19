// Split-precision grouped complex GEMM on the 5th-generation tensor cores
// (tcgen05.mma kind::tf32, accumulators in TMEM, operands staged by TMA).
//
// Every complex operand X is held as four FP32 planes
//   re_hi, re_lo, im_hi, im_lo   (hi = x rounded to TF32, lo = x - hi rounded to TF32)
// in one allocation (plane stride P).  A complex product is accumulated as
//   Re += Ah_r Bh_r + Ah_r Bl_r + Al_r Bh_r - (Ah_i Bh_i + Ah_i Bl_i + Al_i Bh_i)
//   Im += Ah_r Bh_i + Ah_r Bl_i + Al_r Bh_i +  Ah_i Bh_r + Ah_i Bl_r + Al_i Bh_r
// i.e. 12 MMAs of 128 x N x 8 per k-step, FP32 accumulation, the minus sign
// carried by the instruction descriptor's negate-A bit.  Both operands are
// K-major (C[m,n] = sum_k A[m,k] B[n,k]); each operand block has its own 3-D
// tensor map (K, rows, 4 planes) and one TMA load brings all four planes of a
// 128-row x 16-column tile (SWIZZLE_64B).  Mode 2 (stage 2 of the matvec)
// takes its A operand, the stage-1 intermediate T, as the raw FP32
// accumulator in two planes: four converter warps load it and write the four
// TF32 planes into shared memory in the same swizzled layout, which halves
// T's HBM traffic in both stages.
//
// The split-BF16 form (modes 3 and 4) keeps the same pipeline with BF16
// operand planes re_hi, re_mid, im_hi, im_mid (hi = x rounded to BF16, mid =
// x - hi rounded to BF16) and tcgen05.mma kind::f16 with BF16 inputs: 12
// MMAs of 128 x N x 16 per 16-wide k-step, the same three products per real
// product.  A 64-byte shared-memory row holds 32 BF16 K columns, so a stage
// covers twice the K of the TF32 form for the same bytes, and each MMA runs
// at twice the TF32 rate.  Stage 1 (mode 3) writes T split into four BF16
// planes, so stage 2 (mode 4) reads it by TMA like any other operand; the
// canonical-order form (canonical_tc.cu) chains three mode-3 launches and a
// mode-4 one the same way.  A plan may opt narrow tiles (N <= 32) into the
// four-plane form: one MMA per A plane against all four B planes at once
// (N' = 4N), 4 MMAs instead of 12, combined in the epilogue.
//
// Persistent: one CTA per SM walks a list of 128 x N (N <= 128) output tiles
// (tile i of CTA b is tiles[b + i * gridDim]; the host orders them by
// decreasing work, or row tile by row tile within groups that share A),
// each the K-concatenation of its task's terms.  Warp 0 issues TMA loads
// into a 3-stage ring and runs ahead across tile boundaries (its lanes load
// the next 32 tiles' records at once), warp 1 issues the MMAs into one of two
// TMEM accumulator buffers, warps 2-5 (2-9 in mode 3) drain the other buffer
// and write the output (mode 3 through a shared-memory box per warp, in
// 16-byte runs), so the epilogue of a tile overlaps the loads and MMAs of the
// next.  Every mbarrier wait is bounded: on time-out the kernel raises an
// error word, skips the remaining work, frees its TMEM and returns.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include <cuda_bf16.h>

#include "tc_gemm.h"
#include "tf32_round.cuh"

namespace cmps {
namespace tc {

// Modes: 1 TF32, A by TMA, FP32 output (two planes); 2 TF32, A from two
// FP32 planes through the converter warps, FP64 output; 3 BF16, A by TMA,
// output split into four BF16 planes; 4 BF16, A by TMA, FP64 output.
// Warps 0 producer, 1 MMA, 2-5 epilogue; mode 2 adds warps 6-9, which load
// the A tiles from global memory and split them into TF32 planes.
// epilogue warps per TMEM lane quadrant: mode 3 splits every accumulator
// into four BF16 planes, so warps 6-9 join 2-5 (two per quadrant, taking
// 16-column chunks in turn)
template <int MODE>
__host__ __device__ constexpr int epi_per_quad() {
  return MODE == 3 ? 2 : 1;
}
template <int MODE>
__host__ __device__ constexpr int epilogue_warps() {
  return 4 * epi_per_quad<MODE>();
}
template <int MODE>
__host__ __device__ constexpr int threads_of() {
  return MODE == 2 ? 320 : 32 * (2 + epilogue_warps<MODE>());
}
template <int MODE>
__host__ __device__ constexpr bool bf16_mode() {
  return MODE >= 3;
}
template <int MODE>
__host__ __device__ constexpr bool tma_a() {
  return MODE != 2;
}
// the four-plane MMA form of a narrow BF16 tile (TcTile::wide, set by the
// host for N <= 32 with B planes of exactly N rows: 8N TMEM columns)
template <int MODE>
__device__ __forceinline__ bool wide_tile(const TcTile& t) {
  return bf16_mode<MODE>() && t.wide && t.nmma <= 32 && t.b_rows == t.nmma;
}
constexpr int kStages = 3;
constexpr int kBN = 128, kBK = 16;  // TF32 k-step; a BF16 k-step is 2 kBK wide
constexpr int kPlaneTileBytes = 128 * kBK * 4;          // 8 KB: 128 rows x 64 B
constexpr int kOperandBytes = 4 * kPlaneTileBytes;      // 32 KB: four planes
constexpr int kStageBytes = 2 * kOperandBytes;          // A + B
constexpr int kSmemBytes = kStages * kStageBytes + 1024 /*align*/ + 256 /*barriers*/;
// Mode 3 stages its output through shared memory: per epilogue warp one
// 32-row x 16-column x 4-plane BF16 box (rows innermost, 4 KB), after the
// barriers.
constexpr int kStoreBoxBytes = 32 * 16 * 4 * 2;
template <int MODE>
__host__ __device__ constexpr int smem_bytes_of() {
  return kSmemBytes + (MODE == 3 ? epilogue_warps<3>() * kStoreBoxBytes : 0);
}
static_assert(smem_bytes_of<3>() <= 232448, "shared memory per CTA");
constexpr uint32_t kTmemCols = 512;                      // two buffers of {Re at +0, Im at +128}
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s per wait

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait (wall-clock limit): returns false, and raises *err, when the
// limit is reached or another CTA already raised it.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, int code) {
  const unsigned long long t0 = now_ns();
  while (!mbar_try(bar, parity)) {
    if (now_ns() - t0 > kWaitLimitNs) {
      atomicExch(err, code);
      return false;
    }
    if (*(volatile int*)err) return false;
  }
  return true;
}

// The tensor maps live in global memory, written by a host copy before the
// launch.  A freed plan's maps can leave descriptors cached for an address
// that a later plan reuses, so the issuing thread orders its TMA reads of a
// map after the generic-proxy write with an acquire fence on that map.
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.sys [%0], 128;" ::"l"((uint64_t)map) : "memory");
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(smem_u32(dst)), "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void sts16(uint32_t addr, uint32_t v) {
  asm volatile("st.shared.u16 [%0], %1;" ::"r"(addr), "h"((unsigned short)v) : "memory");
}

// UMMA shared-memory descriptor, K-major, SWIZZLE_64B: 64-byte rows, 8-row
// groups 512 B apart (SBO), version 1.
__device__ __forceinline__ uint64_t smem_desc_sw64(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr & 0x3FFFF) >> 4);
  d |= (uint64_t)1 << 16;             // LBO (unused for swizzled K-major)
  d |= (uint64_t)(512 >> 4) << 32;    // SBO
  d |= (uint64_t)1 << 46;             // version
  d |= (uint64_t)4 << 61;             // SWIZZLE_64B
  return d;
}

// Instruction descriptor: kind::tf32, D f32, A/B tf32, K-major, M = 128.
__device__ __forceinline__ uint32_t idesc_tf32(int n, bool neg_a) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((neg_a ? 1u : 0u) << 13) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
// Instruction descriptor: kind::f16, D f32, A/B bf16, K-major, M = 128.
__device__ __forceinline__ uint32_t idesc_bf16(int n, bool neg_a) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((neg_a ? 1u : 0u) << 13) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

// tcgen05.ld of 16 columns without the wait: the registers are written
// asynchronously and may be read only after tmem_wait(r) on them
__device__ __forceinline__ void tmem_ld16_issue(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
// wait for the outstanding tcgen05.ld; the registers pass through the asm so
// that no read of them moves above the wait
__device__ __forceinline__ void tmem_wait(uint32_t* a, uint32_t* b) {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
  asm volatile("" : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]),
               "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]));
  asm volatile("" : "+r"(b[0]), "+r"(b[1]), "+r"(b[2]), "+r"(b[3]), "+r"(b[4]), "+r"(b[5]), "+r"(b[6]), "+r"(b[7]),
               "+r"(b[8]), "+r"(b[9]), "+r"(b[10]), "+r"(b[11]), "+r"(b[12]), "+r"(b[13]), "+r"(b[14]), "+r"(b[15]));
}

template <int MODE>
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  if (bf16_mode<MODE>())
    umma_bf16(tmem_d, a, b, idesc, acc);
  else
    umma_tf32(tmem_d, a, b, idesc, acc);
}

// {bf16(hi_half), bf16(lo_half)} packed, round to nearest
__device__ __forceinline__ uint32_t bf16x2(float hi_half, float lo_half) {
  uint32_t d;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi_half), "f"(lo_half));
  return d;
}

// hi = x rounded to BF16, mid = x - hi rounded to BF16 (raw bits)
__device__ __forceinline__ void bf16_split(float x, uint16_t* hi, uint16_t* mid) {
  const __nv_bfloat16 h = __float2bfloat16_rn(x);
  const __nv_bfloat16 m = __float2bfloat16_rn(x - __bfloat162float(h));
  *hi = __bfloat16_as_ushort(h);
  *mid = __bfloat16_as_ushort(m);
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

template <int MODE>
__global__ void __launch_bounds__(threads_of<MODE>(), 1)
tc_split_gemm(const TcTile* __restrict__ tiles, int ntiles, const TcTask* __restrict__ tasks,
              const TcTerm* __restrict__ terms, const CUtensorMap* __restrict__ amaps,
              const CUtensorMap* __restrict__ bmaps, const TcADesc* __restrict__ adescs,
              const float* __restrict__ ain, int64_t a_plane, float* __restrict__ out32, int64_t out32_plane,
              double* __restrict__ out64, int64_t out64_plane, int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* full = (uint64_t*)(smem + kStages * kStageBytes);
  uint64_t* empty = full + kStages;
  uint64_t* tfull = empty + kStages;   // [2]: accumulator buffer ready for the epilogue
  uint64_t* tempty = tfull + 2;        // [2]: accumulator buffer drained by the epilogue
  uint32_t* tmem_slot = (uint32_t*)(tempty + 2);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], MODE == 2 ? 5 : 1);  // mode 2: the B copy plus one arrival per converter warp
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], epilogue_warps<MODE>());  // one arrival per epilogue warp
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    // ---------------- TMA producer: runs ahead across tile boundaries ----------------
    // The records of this CTA's next 32 tiles (origin, B box rows, term
    // range and first term) are loaded by the 32 lanes at once and handed to
    // lane 0 by shuffles, so the dependent loads tile -> task -> term cost one
    // round of latency per 32 tiles, not one per tile (a tile of one k-step
    // would otherwise leave the ring empty while lane 0 waits on them).
    // Lane 0 issues the copies and fetches each next term of a tile while
    // the current one's copies go out.  `ok` is warp-uniform.
    int it = 0;  // global iteration counter of this CTA (lane 0)
    bool ok = true;
    const int grid = (int)gridDim.x;
    for (int base = blockIdx.x; base < ntiles && ok; base += 32 * grid) {
      const int my = base + lane * grid;
      int m0 = 0, n0 = 0, brows = 0, t0 = 0, t1 = 0;
      TcTerm f{};
      if (my < ntiles) {
        const TcTile tl = tiles[my];
        m0 = tl.m0;
        n0 = tl.n0;
        brows = tl.b_rows;
        t0 = tasks[tl.task].t0;
        t1 = tasks[tl.task].t1;
        if (t1 > t0) f = terms[t0];
      }
      const int cnt = min(32, (ntiles - base + grid - 1) / grid);
      for (int j = 0; j < cnt; ++j) {
        const int jm0 = __shfl_sync(0xffffffffu, m0, j), jn0 = __shfl_sync(0xffffffffu, n0, j);
        const int jb = __shfl_sync(0xffffffffu, brows, j);
        const int jt0 = __shfl_sync(0xffffffffu, t0, j), jt1 = __shfl_sync(0xffffffffu, t1, j);
        TcTerm tm;
        tm.a_map = __shfl_sync(0xffffffffu, f.a_map, j);
        tm.b_map = __shfl_sync(0xffffffffu, f.b_map, j);
        tm.a_x0 = __shfl_sync(0xffffffffu, f.a_x0, j);
        tm.k = __shfl_sync(0xffffffffu, f.k, j);
        tm.a_y0 = __shfl_sync(0xffffffffu, f.a_y0, j);
        if (lane == 0) {
          for (int t = jt0; t < jt1 && ok; ++t) {
            TcTerm nx{};
            if (t + 1 < jt1) nx = terms[t + 1];  // in flight during this term's copies
            if (tma_a<MODE>()) tensormap_acquire(amaps + tm.a_map);
            tensormap_acquire(bmaps + tm.b_map);
            constexpr int kStep = bf16_mode<MODE>() ? 2 * kBK : kBK;  // K columns per 64-byte row
            for (int k0 = 0; k0 < tm.k; k0 += kStep, ++it) {
              const int s = it % kStages;
              const uint32_t ph = (uint32_t)((it / kStages) & 1);
              if (!mbar_wait(&empty[s], ph ^ 1u, err, 1)) {
                ok = false;
                break;
              }
              uint8_t* sa = smem + s * kStageBytes;
              uint8_t* sb = sa + kOperandBytes;
              // A: 128-row box (mode 1; written by the converter warps in mode 2);
              // B: the task's b_rows-row box; both four planes
              const uint32_t bbytes = 4u * 64u * (uint32_t)jb;
              mbar_expect_tx(&full[s], (tma_a<MODE>() ? (uint32_t)kOperandBytes : 0u) + bbytes);
              if (tma_a<MODE>()) tma_load_3d(sa, amaps + tm.a_map, tm.a_x0 + k0, jm0 + tm.a_y0, 0, &full[s]);
              tma_load_3d(sb, bmaps + tm.b_map, k0, jn0, 0, &full[s]);
            }
            tm = nx;
          }
        }
        ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
        if (!ok) break;
      }
    }
    if (lane == 0 && !ok) {
      // let the copies already in flight land before the CTA exits
      for (int j = max(0, it - kStages); j < it; ++j) {
        const unsigned long long t0w = now_ns();
        while (!mbar_try(&full[j % kStages], (uint32_t)((j / kStages) & 1)) && now_ns() - t0w < kWaitLimitNs) {
        }
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      int it = 0, tc = 0;
      bool ok = true;
      TcTile nxt = blockIdx.x < (unsigned)ntiles ? tiles[blockIdx.x] : TcTile{};
      for (int ti = blockIdx.x; ti < ntiles && ok; ti += gridDim.x, ++tc) {
        const TcTile tile = nxt;
        if (ti + (int)gridDim.x < ntiles) nxt = tiles[ti + gridDim.x];  // in flight during this tile
        const int nmma = tile.nmma;  // multiple of 16 for M = 128
        // A narrow BF16 tile (N <= 32) in a plan that opts in runs the
        // four-plane form: the B planes re_hi, re_mid, im_hi, im_mid lie back
        // to back in shared memory (b_rows = N rows each), so one MMA per A
        // plane with N' = 4N forms every product of that plane; (A_hi +
        // A_mid) . B_plane accumulates per plane block: 4 MMAs of 4N instead
        // of 12 of N.
        const bool wide = wide_tile<MODE>(tile);
        const int nw = wide ? 4 * nmma : nmma;
        const uint32_t id_pos = bf16_mode<MODE>() ? idesc_bf16(nw, false) : idesc_tf32(nw, false);
        const uint32_t id_neg = bf16_mode<MODE>() ? idesc_bf16(nw, true) : idesc_tf32(nw, true);
        const int buf = tc & 1;
        const uint32_t use = (uint32_t)(tc >> 1);
        if (!mbar_wait(&tempty[buf], (use & 1u) ^ 1u, err, 4)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t d_re = tmem + (uint32_t)(buf * 256), d_im = d_re + 128;
        const uint32_t b_plane = 64u * (uint32_t)tile.b_rows;  // bytes per B plane in shared memory
        bool first = true;
        {
          for (int kst = 0; kst < tile.kiters; ++kst, ++it) {
            const int s = it % kStages;
            const uint32_t ph = (uint32_t)((it / kStages) & 1);
            if (!mbar_wait(&full[s], ph, err, 2)) {
              ok = false;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = smem_u32(smem + s * kStageBytes);
            const uint32_t b0 = a0 + kOperandBytes;
#pragma unroll
            for (int kk = 0; kk < kBK / 8; ++kk) {
              // planes: 0 re_hi, 1 re_lo, 2 im_hi, 3 im_lo
              uint64_t A[4], B[4];
#pragma unroll
              for (int p = 0; p < 4; ++p) {
                A[p] = smem_desc_sw64(a0 + p * kPlaneTileBytes + kk * 32);
                B[p] = smem_desc_sw64(b0 + p * b_plane + kk * 32);
              }
              const uint32_t acc = first ? 0u : 1u;
              first = false;
              if (wide) {
                // d_re = (A_re_hi + A_re_mid) . [B_re_hi | B_re_mid | B_im_hi | B_im_mid], d_im likewise
                umma<MODE>(d_re, A[0], B[0], id_pos, acc);
                umma<MODE>(d_re, A[1], B[0], id_pos, 1u);
                umma<MODE>(d_im, A[2], B[0], id_pos, acc);
                umma<MODE>(d_im, A[3], B[0], id_pos, 1u);
                continue;
              }
              // planes 1 and 3 are lo (TF32) or mid (BF16)
              umma<MODE>(d_re, A[0], B[0], id_pos, acc);
              umma<MODE>(d_re, A[0], B[1], id_pos, 1u);
              umma<MODE>(d_re, A[1], B[0], id_pos, 1u);
              umma<MODE>(d_re, A[2], B[2], id_neg, 1u);
              umma<MODE>(d_re, A[2], B[3], id_neg, 1u);
              umma<MODE>(d_re, A[3], B[2], id_neg, 1u);
              umma<MODE>(d_im, A[0], B[2], id_pos, acc);
              umma<MODE>(d_im, A[0], B[3], id_pos, 1u);
              umma<MODE>(d_im, A[1], B[2], id_pos, 1u);
              umma<MODE>(d_im, A[2], B[0], id_pos, 1u);
              umma<MODE>(d_im, A[2], B[1], id_pos, 1u);
              umma<MODE>(d_im, A[3], B[0], id_pos, 1u);
            }
            umma_commit(&empty[s]);
          }
        }
        umma_commit(&tfull[buf]);  // arrives at once for a tile without terms
      }
    }
  } else if (MODE == 2 && warp >= 6) {
    // ---------------- A converters (mode 2): warps 6..9, one A row per thread ----------------
    // Each k-step: this row's 16 K columns of the re and im planes are loaded,
    // split into TF32 hi / lo and stored into the four A planes of the slot in
    // the SWIZZLE_64B K-major layout the MMA descriptors read (16-byte chunk c
    // of row r at r * 64 + ((c ^ ((r >> 1) & 3)) << 4)), made visible to the
    // tensor core's async proxy and signalled on the slot's full barrier.  A
    // cursor over this CTA's k-steps (tile, term, k0) runs one step ahead of
    // the stores, so each row's global load is in flight while the previous
    // k-step is converted and waits for its slot.
    const int row = (warp - 6) * 32 + lane;
    const uint32_t sw = (uint32_t)((row >> 1) & 3);
    struct Cur {
      int ti, t, t1, k0, k, a_x0, m0;
      TcADesc ad;
      bool valid;
    };
    auto first_term = [&](Cur& c) {
      // from term c.t of tile c.ti onwards, skipping tiles without terms
      while (c.valid && c.t >= c.t1) {
        c.ti += gridDim.x;
        if (c.ti >= ntiles) {
          c.valid = false;
          return;
        }
        const TcTile tl = tiles[c.ti];
        const TcTask tk = tasks[tl.task];
        c.m0 = tl.m0;
        c.t = tk.t0;
        c.t1 = tk.t1;
      }
      if (!c.valid) return;
      const TcTerm tm = terms[c.t];
      c.ad = adescs[tm.a_map];
      c.k = tm.k;
      c.a_x0 = tm.a_x0;
      c.k0 = 0;
    };
    auto advance = [&](Cur& c) {
      c.k0 += kBK;
      if (c.k0 < c.k) return;
      ++c.t;
      first_term(c);
    };
    auto load = [&](const Cur& c, float* xr, float* xi) {
      const int gr = c.m0 + row;
      const bool rok = gr < c.ad.rows;
      const float* pre = ain + c.ad.off + (int64_t)(rok ? gr : 0) * c.ad.ld;
      const float* pim = pre + a_plane;
      const int x0 = c.a_x0 + c.k0;
      if (rok && x0 + 16 <= c.ad.cols) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float4 a = *(const float4*)(pre + x0 + 4 * q);
          const float4 b = *(const float4*)(pim + x0 + 4 * q);
          xr[4 * q] = a.x; xr[4 * q + 1] = a.y; xr[4 * q + 2] = a.z; xr[4 * q + 3] = a.w;
          xi[4 * q] = b.x; xi[4 * q + 1] = b.y; xi[4 * q + 2] = b.z; xi[4 * q + 3] = b.w;
        }
      } else {
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const bool in = rok && x0 + q < c.ad.cols;
          xr[q] = in ? pre[x0 + q] : 0.f;
          xi[q] = in ? pim[x0 + q] : 0.f;
        }
      }
    };
    Cur cur;
    cur.ti = (int)blockIdx.x - (int)gridDim.x;  // first_term steps to this CTA's first tile
    cur.t = cur.t1 = 0;
    cur.valid = true;
    first_term(cur);
    float ar[16], ai[16], br[16], bi[16];
    if (cur.valid) load(cur, ar, ai);
    int it = 0;
    while (cur.valid) {
      Cur nxt = cur;
      advance(nxt);
      if (nxt.valid) load(nxt, br, bi);  // next k-step's row, in flight during this one
      const int s = it % kStages;
      const uint32_t ph = (uint32_t)((it / kStages) & 1);
      int go = 1;
      if (lane == 0) go = mbar_wait(&empty[s], ph ^ 1u, err, 5) ? 1 : 0;
      go = __shfl_sync(0xffffffffu, go, 0);
      if (!go) break;
      uint8_t* sa = smem + s * kStageBytes + row * 64;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        float4 h_r, l_r, h_i, l_i;
        float* hr = &h_r.x; float* lr = &l_r.x; float* hi = &h_i.x; float* li = &l_i.x;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float a = ar[4 * q + e], b = ai[4 * q + e];
          hr[e] = tf32_rna(a);
          lr[e] = tf32_rna(a - hr[e]);
          hi[e] = tf32_rna(b);
          li[e] = tf32_rna(b - hi[e]);
        }
        const uint32_t off = ((uint32_t)q ^ sw) << 4;
        *(float4*)(sa + 0 * kPlaneTileBytes + off) = h_r;
        *(float4*)(sa + 1 * kPlaneTileBytes + off) = l_r;
        *(float4*)(sa + 2 * kPlaneTileBytes + off) = h_i;
        *(float4*)(sa + 3 * kPlaneTileBytes + off) = l_i;
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&full[s])) : "memory");
      ++it;
      cur = nxt;
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        ar[q] = br[q];
        ai[q] = bi[q];
      }
    }
  } else if ((warp >= 2 && warp < 6) || (MODE == 3 && warp >= 6)) {
    // ---------------- epilogue: warps 2..5 (and 6..9 in mode 3) ----------------
    const int quad = warp & 3;  // TMEM lane quadrant this warp may access
    const int row = quad * 32 + lane;
    int tc = 0;
    // mode 3, vector-store path: this warp's staging box
    const uint32_t stg = smem_u32(smem + kStages * kStageBytes + 256) + (uint32_t)((warp - 2) * kStoreBoxBytes);
    // the next tile's records are loaded while this tile waits and drains
    TcTile nt = blockIdx.x < (unsigned)ntiles ? tiles[blockIdx.x] : TcTile{};
    TcTask nk = blockIdx.x < (unsigned)ntiles ? tasks[nt.task] : TcTask{};
    for (int ti = blockIdx.x; ti < ntiles; ti += gridDim.x, ++tc) {
      const TcTile tile = nt;
      const TcTask task = nk;
      if (ti + (int)gridDim.x < ntiles) {
        nt = tiles[ti + gridDim.x];
        nk = tasks[nt.task];
      }
      const int ntile = min(kBN, task.n - tile.n0);
      const int nmma = tile.nmma;
      const int buf = tc & 1;
      const uint32_t use = (uint32_t)(tc >> 1);
      int have = task.t1 > task.t0 ? 1 : 0;
      int alive = 1;
      if (lane == 0) {
        if (!mbar_wait(&tfull[buf], use & 1u, err, 3)) alive = 0;
        if (*(volatile int*)err) alive = 0;
      }
      alive = __shfl_sync(0xffffffffu, alive, 0);  // warp-uniform: tcgen05.ld is warp-collective
      if (!alive) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int gm = tile.m0 + row;
      const bool row_ok = gm < task.m;
      const uint32_t tbase = tmem + (uint32_t)(buf * 256) + ((uint32_t)(quad * 32) << 16);
      // mode 3: the warps of a quadrant take 16-column chunks in turn
      const int c_first = 16 * ((warp - 2) / 4);
      const int c_step = 16 * epi_per_quad<MODE>();
      // TMEM loads run one chunk ahead: chunk c + c_step is in flight while
      // chunk c is stored (every lane issues and waits; tcgen05.ld is
      // warp-collective, so the row check comes after)
      uint32_t ra[16], ia[16];
      const bool wide = wide_tile<MODE>(tile);
      if (have && !wide && c_first < nmma) {
        tmem_ld16_issue(tbase + c_first, ra);
        tmem_ld16_issue(tbase + 128 + c_first, ia);
      }
      for (int c = c_first; c < nmma; c += c_step) {
        float vr[16], vi[16];
        if (have && wide) {
          // four-plane form: block q of d_re / d_im (columns q N ..) holds
          // A_re . B_q / A_im . B_q for B planes re_hi, re_mid, im_hi, im_mid
          //   re = d_re[0] + d_re[1] - d_im[2] - d_im[3]
          //   im = d_re[2] + d_re[3] + d_im[0] + d_im[1]
          tmem_ld16_issue(tbase + c, ra);
          tmem_ld16_issue(tbase + nmma + c, ia);
          tmem_wait(ra, ia);
#pragma unroll
          for (int i = 0; i < 16; ++i) vr[i] = __uint_as_float(ra[i]) + __uint_as_float(ia[i]);
          tmem_ld16_issue(tbase + 128 + 2 * nmma + c, ra);
          tmem_ld16_issue(tbase + 128 + 3 * nmma + c, ia);
          tmem_wait(ra, ia);
#pragma unroll
          for (int i = 0; i < 16; ++i) vr[i] -= __uint_as_float(ra[i]) + __uint_as_float(ia[i]);
          tmem_ld16_issue(tbase + 2 * nmma + c, ra);
          tmem_ld16_issue(tbase + 3 * nmma + c, ia);
          tmem_wait(ra, ia);
#pragma unroll
          for (int i = 0; i < 16; ++i) vi[i] = __uint_as_float(ra[i]) + __uint_as_float(ia[i]);
          tmem_ld16_issue(tbase + 128 + c, ra);
          tmem_ld16_issue(tbase + 128 + nmma + c, ia);
          tmem_wait(ra, ia);
#pragma unroll
          for (int i = 0; i < 16; ++i) vi[i] += __uint_as_float(ra[i]) + __uint_as_float(ia[i]);
        } else if (have) {
          tmem_wait(ra, ia);
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            vr[i] = __uint_as_float(ra[i]);
            vi[i] = __uint_as_float(ia[i]);
          }
          if (c + c_step < nmma) {
            tmem_ld16_issue(tbase + c + c_step, ra);
            tmem_ld16_issue(tbase + 128 + c + c_step, ia);
          }
        } else {
#pragma unroll
          for (int i = 0; i < 16; ++i) vr[i] = vi[i] = 0.f;
        }
        if (MODE == 3 && task.vstore) {
          // Vector-store path, for a chunk inside one column segment: the
          // chunk is split and written by every lane as its row of a
          // [plane][column][row] box in shared memory, then read back as
          // 16-byte runs of 8 rows and stored: lane l takes columns l / 4
          // and 8 + l / 4, rows 8 (l % 4) .. +7, in the four planes.  Rows
          // past the task (whole 8-row runs: its M is a multiple of 8) are
          // not stored.
          const int cnt = min(16, ntile - c);
          const int colA = tile.n0 + c, colB = colA + cnt - 1;
          const int qa = (colA >= task.seg_n0[1]) + (colA >= task.seg_n0[2]) + (colA >= task.seg_n0[3]);
          const int qb = (colB >= task.seg_n0[1]) + (colB >= task.seg_n0[2]) + (colB >= task.seg_n0[3]);
          const int row0 = tile.m0 + quad * 32;
          if (cnt > 0 && qa == qb && row0 < task.m) {
            const int n0 = qa == 0 ? 0 : qa == 1 ? task.seg_n0[1] : qa == 2 ? task.seg_n0[2] : task.seg_n0[3];
            const int64_t so = qa == 0 ? task.seg_off[0] : qa == 1 ? task.seg_off[1] : qa == 2 ? task.seg_off[2]
                                                                                            : task.seg_off[3];
            const int lc = lane >> 2, lr = (lane & 3) * 8;
            const bool rok8 = row0 + lr < task.m;
            uint16_t* g = reinterpret_cast<uint16_t*>(out32) + so + row0 + lr +
                          (int64_t)(colA - n0 + lc) * task.col_stride;
            const uint32_t box = stg + (uint32_t)(lane * 2);
            const uint32_t rd = stg + (uint32_t)(lc * 64 + lr * 2);
            __syncwarp();  // the previous chunk's reads of the box are done
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              const float xr = vr[i], xi = vi[i];
              const uint32_t h2 = bf16x2(xi, xr);
              const float rh = __uint_as_float(h2 << 16), ih = __uint_as_float(h2 & 0xffff0000u);
              const uint32_t m2 = bf16x2(xi - ih, xr - rh);
              sts16(box + (uint32_t)((0 * 16 + i) * 64), h2);
              sts16(box + (uint32_t)((1 * 16 + i) * 64), m2);
              sts16(box + (uint32_t)((2 * 16 + i) * 64), h2 >> 16);
              sts16(box + (uint32_t)((3 * 16 + i) * 64), m2 >> 16);
            }
            __syncwarp();
            uint4 v[2][4];
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
              for (int j = 0; j < 4; ++j)
                asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
                             : "=r"(v[h][j].x), "=r"(v[h][j].y), "=r"(v[h][j].z), "=r"(v[h][j].w)
                             : "r"(rd + (uint32_t)((j * 16 + h * 8) * 64)));
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              if (!rok8 || h * 8 + lc >= cnt) continue;
              uint16_t* gh = g + (int64_t)(h * 8) * task.col_stride;
#pragma unroll
              for (int j = 0; j < 4; ++j) *reinterpret_cast<uint4*>(gh + j * out32_plane) = v[h][j];
            }
            continue;
          }
        }
        if (!row_ok) continue;
        if (MODE == 3) {
          // Fast path: a chunk whose 16 columns lie in one segment (the
          // usual case) stores from one base pointer; re and im are split
          // together with packed conversions: h2 = {hi_im, hi_re}, m2 =
          // {mid_im, mid_re}.
          const int cnt = min(16, ntile - c);
          const int colA = tile.n0 + c, colB = colA + cnt - 1;
          const int qa = (colA >= task.seg_n0[1]) + (colA >= task.seg_n0[2]) + (colA >= task.seg_n0[3]);
          const int qb = (colB >= task.seg_n0[1]) + (colB >= task.seg_n0[2]) + (colB >= task.seg_n0[3]);
          if (cnt > 0 && qa == qb) {
            int64_t so = task.seg_off[0];
            int n0 = 0;
            if (qa == 1) so = task.seg_off[1], n0 = task.seg_n0[1];
            if (qa == 2) so = task.seg_off[2], n0 = task.seg_n0[2];
            if (qa == 3) so = task.seg_off[3], n0 = task.seg_n0[3];
            uint16_t* b0 = reinterpret_cast<uint16_t*>(out32) + so + (int64_t)gm * task.row_stride +
                           (int64_t)(colA - n0) * task.col_stride;
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              if (i >= cnt) break;
              const uint32_t h2 = bf16x2(vi[i], vr[i]);
              const float rh = __uint_as_float(h2 << 16), ih = __uint_as_float(h2 & 0xffff0000u);
              const uint32_t m2 = bf16x2(vi[i] - ih, vr[i] - rh);
              uint16_t* q = b0 + (int64_t)i * task.col_stride;
              q[0] = (uint16_t)h2;
              q[out32_plane] = (uint16_t)m2;
              q[2 * out32_plane] = (uint16_t)(h2 >> 16);
              q[3 * out32_plane] = (uint16_t)(m2 >> 16);
            }
            continue;
          }
        }
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int j = c + i;
          if (j >= ntile) break;
          // the column's segment by selects (an indexed read of the task's
          // arrays would put the task in local memory)
          const int col = tile.n0 + j;
          int64_t so = task.seg_off[0];
          int n0 = 0;
          if (col >= task.seg_n0[1]) so = task.seg_off[1], n0 = task.seg_n0[1];
          if (col >= task.seg_n0[2]) so = task.seg_off[2], n0 = task.seg_n0[2];
          if (col >= task.seg_n0[3]) so = task.seg_off[3], n0 = task.seg_n0[3];
          const int64_t o = so + (int64_t)gm * task.row_stride + (int64_t)(col - n0) * task.col_stride;
          if (MODE == 1) {
            // stage-1 output: the FP32 accumulator, re and im planes (the
            // stage-2 converter warps split it into TF32 hi / lo)
            out32[o] = vr[i];
            out32[o + out32_plane] = vi[i];
          } else if (MODE == 3) {
            // stage-1 output split into BF16 planes re_hi, re_mid, im_hi, im_mid
            uint16_t* o16 = reinterpret_cast<uint16_t*>(out32);
            bf16_split(vr[i], o16 + o, o16 + o + out32_plane);
            bf16_split(vi[i], o16 + o + 2 * out32_plane, o16 + o + 3 * out32_plane);
          } else {
            out64[o] = (double)vr[i];
            out64[o + out64_plane] = (double)vi[i];
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&tempty[buf])) : "memory");
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
  }
}

int smem_bytes() { return kSmemBytes; }

int launch(int mode, const TcPlan& p, float* out32, int64_t out32_plane, double* out64, int64_t out64_plane,
           const float* ain, int64_t a_plane, int* d_err, cudaStream_t st) {
  if (p.tiles.empty()) return CMPS_OK;
  if (p.tiles.size() > 0x7fffffffull) return fail(CMPS_ERR_ARG, "too many tcgen05 tiles");
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int ntiles = (int)p.tiles.size();
  const unsigned grid = (unsigned)std::min(ntiles, sms);
  if (mode == 1 || mode == 3 || mode == 4) {
    if (!p.d_amaps) return fail(CMPS_ERR_STATE, "tcgen05: no A tensor maps");
    auto kern = mode == 1 ? tc_split_gemm<1> : mode == 3 ? tc_split_gemm<3> : tc_split_gemm<4>;
    const int smem = mode == 3 ? smem_bytes_of<3>() : kSmemBytes;
    CMPS_TRY(ensure_smem_optin((const void*)kern, smem));
    const int threads = mode == 3 ? threads_of<3>() : threads_of<1>();
    kern<<<grid, threads, smem, st>>>(p.d_tiles, ntiles, p.d_tasks, p.d_terms, p.d_amaps, p.d_bmaps, nullptr,
                                            nullptr, 0, out32, out32_plane, out64, out64_plane, d_err);
  } else if (mode == 2) {
    if (!ain || !p.d_adescs) return fail(CMPS_ERR_STATE, "tcgen05 mode 2: no A operand");
    CMPS_TRY(ensure_smem_optin((const void*)tc_split_gemm<2>, kSmemBytes));
    tc_split_gemm<2><<<grid, threads_of<2>(), kSmemBytes, st>>>(p.d_tiles, ntiles, p.d_tasks, p.d_terms, nullptr,
                                                                 p.d_bmaps, p.d_adescs, ain, a_plane, out32,
                                                                 out32_plane, out64, out64_plane, d_err);
  } else {
    return fail(CMPS_ERR_ARG, "tcgen05: unknown mode");
  }
  CMPS_CUDA(cudaGetLastError());
  return CMPS_OK;
}

}  // namespace tc
}  // namespace cmps
