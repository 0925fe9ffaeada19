// Grouped complex-double GEMM on the FP64 tensor path (DMMA, mma.sync
// m8n8k4 f64) for sm_100a.
//
// One launch runs a whole list of independent output tiles.  Each output
// region ("task") is C = sum over its terms of op(A_t) op(B_t), where every
// term has its own A block, B block and K -- the K-concatenation that turns
// the charge-sector structure of H_eff (sum over MPO indices and physical
// states) into a single accumulation.  Complex operands are stored as two
// planes (re, im) of one allocation; a complex MAC is four real DMMAs.
// Operands are staged global -> shared with 8-byte cp.async (zero-filled
// outside the block), double buffered.  op(A) is A or A^H (A stored K x M),
// op(B) is B or B^H (B stored N x K), all row-major with leading dimensions.
// NSPLIT: the N index of B and C is two-level (GemmTask::n_in), so one task
// can run over several equally strided column ranges, e.g. the rows of
// every state of one charge class, or one column class of every row.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "internal.h"

namespace cmps {

namespace {

// Output tile BM x BN, four warps of 32 x 32 each (WN = BN / 32 across N).
// Shapes: 64 x 64 (square blocks), 32 x 128 (tasks with M <= 32: a charge
// class of 32 states, a small a0 sector) and 128 x 32 (tasks with N <= 32).
// Shared-memory rows are padded to BM + 4 / BN + 4 doubles (= 4 mod 16):
// conflict-free 8-byte fragment reads.
constexpr int BK = 16;
constexpr int NTHREADS = 128;
constexpr int STAGES = 2;
template <int BM, int BN>
struct Tile {
  static_assert(BM % 32 == 0 && BN % 32 == 0 && (BM / 32) * (BN / 32) == 4, "four 32 x 32 warp tiles");
  static constexpr int WN = BN / 32;
  static constexpr int LDA = BM + 4, LDB = BN + 4;
  static constexpr int PLANE_A = BK * LDA, PLANE_B = BK * LDB;  // doubles per plane per stage
  static constexpr int STAGE_DOUBLES = 2 * PLANE_A + 2 * PLANE_B;  // A re, A im, B re, B im
  static constexpr size_t SMEM_BYTES = (size_t)STAGES * STAGE_DOUBLES * sizeof(double);
};

__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, bool pred) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int sz = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }
__device__ __forceinline__ void cp_wait0() { asm volatile("cp.async.wait_group 0;\n" ::); }

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Offset of column n under the two-level N index (NSPLIT), else n.
template <bool NSPLIT>
__device__ __forceinline__ int64_t ncol(int n, int n_in, int ld_out) {
  if (!NSPLIT) return n;
  const int q = n / n_in;
  return (int64_t)q * ld_out + (n - q * n_in);
}

// Issue the cp.async copies of one (term, k-tile) into stage buffer `buf`.
template <int BM, int BN, bool AH, bool BH, bool NSPLIT>
__device__ __forceinline__ void load_stage(double* buf, const GemmTerm& t, int k0, int m0, int n0, int M,
                                           int N, int n_in, const double* __restrict__ Ar,
                                           const double* __restrict__ Ai, const double* __restrict__ Br,
                                           const double* __restrict__ Bi) {
  using T = Tile<BM, BN>;
  double* sAr = buf;
  double* sAi = buf + T::PLANE_A;
  double* sBr = buf + 2 * T::PLANE_A;
  double* sBi = sBr + T::PLANE_B;
  const int tid = threadIdx.x;
  const int K = t.k;
#pragma unroll
  for (int j = 0; j < (BM * BK) / NTHREADS; ++j) {
    int idx = tid + j * NTHREADS;
    int kk, mm;
    if (!AH) { kk = idx % BK; mm = idx / BK; }   // A[m][k]: consecutive threads along k
    else     { kk = idx / BM; mm = idx % BM; }   // A stored [k][m]: along m
    int gm = m0 + mm, gk = k0 + kk;
    bool ok = (gm < M) && (gk < K);
    int64_t o = ok ? (AH ? t.a_off + (int64_t)gk * t.lda + gm : t.a_off + (int64_t)gm * t.lda + gk) : 0;
    cp_async8(sAr + kk * T::LDA + mm, Ar + o, ok);
    cp_async8(sAi + kk * T::LDA + mm, Ai + o, ok);
  }
#pragma unroll
  for (int j = 0; j < (BN * BK) / NTHREADS; ++j) {
    int idx = tid + j * NTHREADS;
    int kk, nn;
    if (!BH) { kk = idx / BN; nn = idx % BN; }   // B[k][n]: along n
    else     { kk = idx % BK; nn = idx / BK; }   // B stored [n][k]: along k
    int gn = n0 + nn, gk = k0 + kk;
    bool ok = (gn < N) && (gk < K);
    int64_t o = ok ? (BH ? t.b_off + (int64_t)gn * t.ldb + gk
                         : t.b_off + (int64_t)gk * t.ldb + ncol<NSPLIT>(gn, n_in, t.ldb_out))
                   : 0;
    cp_async8(sBr + kk * T::LDB + nn, Br + o, ok);
    cp_async8(sBi + kk * T::LDB + nn, Bi + o, ok);
  }
}

template <int BM, int BN, bool AH, bool BH, bool NSPLIT>
__global__ void __launch_bounds__(NTHREADS, 2)
zgemm_grouped_fp64(const GemmTile* __restrict__ tiles, const GemmTask* __restrict__ tasks,
                   const GemmTerm* __restrict__ terms, const double* __restrict__ Ar,
                   const double* __restrict__ Ai, const double* __restrict__ Br,
                   const double* __restrict__ Bi, double* __restrict__ Cr, double* __restrict__ Ci) {
  extern __shared__ double smem[];
  const GemmTile tile = tiles[blockIdx.x];
  const GemmTask task = tasks[tile.task];
  const int m0 = tile.m0, n0 = tile.n0, M = task.m, N = task.n;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  using T = Tile<BM, BN>;
  const int wm = warp / T::WN, wn = warp % T::WN;
  const int gid = lane >> 2, tig = lane & 3;

  double accr[4][4][2], acci[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      accr[i][j][0] = accr[i][j][1] = 0.0;
      acci[i][j][0] = acci[i][j][1] = 0.0;
    }

  // iteration cursor over (term, k-tile)
  int cur_t = task.t0, cur_k = 0;
  int nxt_t = cur_t, nxt_k = 0;
  bool have = cur_t < task.t1;
  if (have) {
    GemmTerm t = terms[cur_t];
    load_stage<BM, BN, AH, BH, NSPLIT>(smem, t, 0, m0, n0, M, N, task.n_in, Ar, Ai, Br, Bi);
    cp_commit();
    nxt_k = BK;
    if (nxt_k >= t.k) { nxt_t = cur_t + 1; nxt_k = 0; }
  }
  int stage = 0;
  while (have) {
    bool more = nxt_t < task.t1;
    if (more) {
      GemmTerm t = terms[nxt_t];
      load_stage<BM, BN, AH, BH, NSPLIT>(smem + (stage ^ 1) * T::STAGE_DOUBLES, t, nxt_k, m0, n0, M, N, task.n_in, Ar,
                                         Ai, Br, Bi);
      cp_commit();
      cp_wait1();
    } else {
      cp_wait0();
    }
    __syncthreads();
    const double* sAr = smem + stage * T::STAGE_DOUBLES;
    const double* sAi = sAr + T::PLANE_A;
    const double* sBr = sAr + 2 * T::PLANE_A;
    const double* sBi = sBr + T::PLANE_B;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double ar[4], ai[4], nai[4], br[4], bi[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        int mm = wm * 32 + i * 8 + gid;
        ar[i] = sAr[(kk + tig) * T::LDA + mm];
        ai[i] = sAi[(kk + tig) * T::LDA + mm];
        if (AH) ai[i] = -ai[i];
        nai[i] = -ai[i];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        int nn = wn * 32 + j * 8 + gid;
        br[j] = sBr[(kk + tig) * T::LDB + nn];
        bi[j] = sBi[(kk + tig) * T::LDB + nn];
        if (BH) bi[j] = -bi[j];
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          dmma(accr[i][j][0], accr[i][j][1], ar[i], br[j]);
          dmma(accr[i][j][0], accr[i][j][1], nai[i], bi[j]);
          dmma(acci[i][j][0], acci[i][j][1], ar[i], bi[j]);
          dmma(acci[i][j][0], acci[i][j][1], ai[i], br[j]);
        }
    }
    __syncthreads();
    // advance
    have = more;
    if (more) {
      cur_t = nxt_t;
      cur_k = nxt_k;
      GemmTerm t = terms[cur_t];
      nxt_k = cur_k + BK;
      nxt_t = cur_t;
      if (nxt_k >= t.k) { nxt_t = cur_t + 1; nxt_k = 0; }
      stage ^= 1;
    }
  }
  // epilogue
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        int gm = m0 + wm * 32 + i * 8 + gid;
        int gn = n0 + wn * 32 + j * 8 + 2 * tig + e;
        if (gm < M && gn < N) {
          int64_t o = task.c_off + (int64_t)gm * task.ldc + ncol<NSPLIT>(gn, task.n_in, task.ldc_out);
          Cr[o] = accr[i][j][e];
          Ci[o] = acci[i][j][e];
        }
      }
}

template <int BM, int BN, bool AH, bool BH, bool NSPLIT>
int launch_variant(const GemmPlan& p, const Planar& A, const Planar& B, Planar& C, cudaStream_t st) {
  using T = Tile<BM, BN>;
  CMPS_TRY(ensure_smem_optin((const void*)zgemm_grouped_fp64<BM, BN, AH, BH, NSPLIT>, (int)T::SMEM_BYTES));
  if (p.tiles.empty()) return CMPS_OK;
  const int64_t ntiles = (int64_t)p.tiles.size();
  if (ntiles > 0x7fffffff) return fail(CMPS_ERR_ARG, "too many GEMM tiles");
  zgemm_grouped_fp64<BM, BN, AH, BH, NSPLIT><<<(unsigned)ntiles, NTHREADS, T::SMEM_BYTES, st>>>(
      p.d_tiles, p.d_tasks, p.d_terms, A.re(), A.im(), B.re(), B.im(), C.re(), C.im());
  CMPS_CUDA(cudaGetLastError());
  return CMPS_OK;
}

template <int BM, int BN>
int launch_shape(const GemmPlan& p, bool a_h, bool b_h, const Planar& A, const Planar& B, Planar& C,
                 cudaStream_t st) {
  if (p.nsplit) {
    if (a_h || b_h) return fail(CMPS_ERR_STATE, "two-level N index with a conjugate-transposed operand");
    return launch_variant<BM, BN, false, false, true>(p, A, B, C, st);
  }
  if (!a_h && !b_h) return launch_variant<BM, BN, false, false, false>(p, A, B, C, st);
  if (a_h && !b_h) return launch_variant<BM, BN, true, false, false>(p, A, B, C, st);
  if (!a_h && b_h) return launch_variant<BM, BN, false, true, false>(p, A, B, C, st);
  return launch_variant<BM, BN, true, true, false>(p, A, B, C, st);
}

constexpr int kShapes[3][2] = {{64, 64}, {32, 128}, {128, 32}};

}  // namespace

int gemm_shape_m(int shape) { return kShapes[shape][0]; }
int gemm_shape_n(int shape) { return kShapes[shape][1]; }

int launch_zgemm_fp64(const GemmPlan& p, bool a_h, bool b_h, const Planar& A, const Planar& B, Planar& C,
                      cudaStream_t st) {
  switch (p.shape) {
    case 0: return launch_shape<64, 64>(p, a_h, b_h, A, B, C, st);
    case 1: return launch_shape<32, 128>(p, a_h, b_h, A, B, C, st);
    case 2: return launch_shape<128, 32>(p, a_h, b_h, A, B, C, st);
    default: return fail(CMPS_ERR_STATE, "GEMM plan not uploaded (no tile shape)");
  }
}

// Tile shape of a plan, chosen from its own tasks: the shape whose padded
// work (every task rounded up to whole tiles, times its K) plus a fixed cost
// per tile (prologue, epilogue, scheduling: the work of 16 k-steps of a
// 32 x 32 quarter tile) is least.  Ties keep 64 x 64.
static int pick_shape(const GemmPlan& p) {
  double best = 0.0;
  int shape = 0;
  for (int s = 0; s < 3; ++s) {
    const int bm = kShapes[s][0], bn = kShapes[s][1];
    double cost = 0.0;
    for (const GemmTask& t : p.tasks) {
      if (t.m <= 0 || t.n <= 0) continue;
      int64_t k = 0;
      for (int q = t.t0; q < t.t1; ++q) k += p.terms[q].k;
      const double tm = (double)((t.m + bm - 1) / bm), tn = (double)((t.n + bn - 1) / bn);
      cost += tm * tn * ((double)bm * bn * (double)std::max<int64_t>(k, BK) + 16.0 * 32 * 32 * BK);
    }
    if (s == 0 || cost < 0.97 * best) {
      best = cost;
      shape = s;
    }
  }
  return shape;
}

int GemmPlan::retile(int s, cudaStream_t st) {
  if (s < 0 || s > 2) return fail(CMPS_ERR_ARG, "GEMM plan: unknown tile shape");
  if (!d_tasks && !tasks.empty()) return fail(CMPS_ERR_STATE, "GEMM plan not uploaded");
  const int bm = kShapes[s][0], bn = kShapes[s][1];
  std::vector<GemmTile> nt;
  for (size_t i = 0; i < tasks.size(); ++i) {
    const GemmTask& t = tasks[i];
    for (int m0 = 0; m0 < t.m; m0 += bm)
      for (int n0 = 0; n0 < t.n; n0 += bn) nt.push_back(GemmTile{(int32_t)i, m0, n0, 0});
  }
  GemmTile* d = nullptr;
  if (!nt.empty()) {
    CMPS_CUDA(dmalloc((void**)&d, nt.size() * sizeof(GemmTile)));
    const int rc = copy_wait(d, nt.data(), nt.size() * sizeof(GemmTile), cudaMemcpyHostToDevice, st);
    if (rc != CMPS_OK) {
      dfree(d);
      return rc;
    }
  }
  if (d_tiles) dfree(d_tiles);
  d_tiles = d;
  tiles.swap(nt);
  shape = s;
  return CMPS_OK;
}

namespace {
std::mutex g_tune_mu;
std::map<std::vector<int64_t>, int> g_tune_cache;  // plan signature -> measured best shape
}  // namespace

int autotune_plan(GemmPlan& p, int role, const std::function<int()>& run, cudaStream_t st, TuneStats* stats) {
  if (p.tasks.empty()) return CMPS_OK;
  // signature: the role, the task and term counts, the flops to 3 digits and
  // the padded-work choice -- plans of the same shape population share it
  double fl = 0.0;
  for (const GemmTask& t : p.tasks)
    for (int q = t.t0; q < t.t1; ++q) fl += 8.0 * t.m * (double)t.n * p.terms[q].k;
  const int64_t fq = fl > 0.0 ? (int64_t)std::llround(std::log10(fl) * 300.0) : 0;
  const std::vector<int64_t> sig{role, (int64_t)p.tasks.size(), (int64_t)p.terms.size(), fq, p.shape};
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune_cache.find(sig);
    if (it != g_tune_cache.end()) {
      if (stats) ++stats->cached;
      return it->second == p.shape ? CMPS_OK : p.retile(it->second, st);
    }
  }
  const int heuristic = p.shape;
  float best = 0.0f, heur = 0.0f;
  int pick = heuristic;
  cudaEvent_t e0, e1;
  CMPS_CUDA(cudaEventCreate(&e0));
  CMPS_CUDA(cudaEventCreate(&e1));
  int rc = CMPS_OK;
  for (int s = 0; s < 3 && rc == CMPS_OK; ++s) {
    rc = p.retile(s, st);
    if (rc == CMPS_OK) rc = run();  // warm-up
    if (rc != CMPS_OK) break;
    cudaEventRecord(e0, st);
    for (int r = 0; r < 3 && rc == CMPS_OK; ++r) rc = run();
    cudaEventRecord(e1, st);
    if (rc != CMPS_OK || cudaEventSynchronize(e1) != cudaSuccess) {
      if (rc == CMPS_OK) rc = fail(CMPS_ERR_CUDA, "autotune: timing failed");
      break;
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (s == heuristic) heur = ms;
    if (s == 0 || ms < best) {
      best = ms;
      pick = s;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CMPS_TRY(rc);
  CMPS_TRY(p.retile(pick, st));
  if (std::getenv("CMPS_TUNE_TRACE"))
    std::fprintf(stderr, "autotune role %d: tasks %zu, heuristic shape %d %.3f ms, best shape %d %.3f ms\n", role,
                 p.tasks.size(), heuristic, heur / 3, pick, best / 3);
  if (stats) {
    ++stats->tuned;
    stats->ms_heuristic += heur / 3;
    stats->ms_best += best / 3;
  }
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tune_cache[sig] = pick;
  return CMPS_OK;
}

int GemmPlan::upload(cudaStream_t st) {
  shape = pick_shape(*this);
  const int bm = kShapes[shape][0], bn = kShapes[shape][1];
  tiles.clear();
  for (size_t i = 0; i < tasks.size(); ++i) {
    const GemmTask& t = tasks[i];
    for (int m0 = 0; m0 < t.m; m0 += bm)
      for (int n0 = 0; n0 < t.n; n0 += bn) tiles.push_back(GemmTile{(int32_t)i, m0, n0, 0});
  }
  release();
  auto up = [st](auto& v, auto** d) -> int {
    if (v.empty()) return CMPS_OK;
    size_t bytes = v.size() * sizeof(v[0]);
    CMPS_CUDA(dmalloc((void**)d, bytes));
    return copy_wait(*d, v.data(), bytes, cudaMemcpyHostToDevice, st);
  };
  CMPS_TRY(up(tasks, &d_tasks));
  CMPS_TRY(up(terms, &d_terms));
  CMPS_TRY(up(tiles, &d_tiles));
  return CMPS_OK;
}

int GemmPlan::validate(bool a_h, bool b_h, int64_t a_len, int64_t b_len, int64_t c_len, const char* what) const {
  for (const GemmTask& t : tasks) {
    if (t.m < 0 || t.n < 0 || t.t0 < 0 || t.t1 < t.t0 || t.t1 > (int32_t)terms.size())
      return fail(CMPS_ERR_STATE, std::string(what) + ": malformed task");
    if (t.m == 0 || t.n == 0) continue;
    if ((t.n_in > 0) != nsplit || (nsplit && (a_h || b_h || t.ldc_out < t.n_in)))
      return fail(CMPS_ERR_STATE, std::string(what) + ": malformed two-level N index");
    // extent of one row of C or B along N: the last column's offset + 1
    const int64_t nspan = nsplit ? (int64_t)((t.n - 1) / t.n_in) * t.ldc_out + (t.n - 1) % t.n_in + 1 : t.n;
    if (t.c_off < 0 || t.c_off + (int64_t)(t.m - 1) * t.ldc + nspan > c_len || (!nsplit && t.ldc < t.n))
      return fail(CMPS_ERR_STATE, std::string(what) + ": output range outside its buffer");
    for (int q = t.t0; q < t.t1; ++q) {
      const GemmTerm& tm = terms[q];
      if (tm.k <= 0) return fail(CMPS_ERR_STATE, std::string(what) + ": empty term");
      // A is M x K (row-major, lda >= K) or stored K x M (lda >= M)
      int64_t arows = a_h ? tm.k : t.m, acols = a_h ? t.m : tm.k;
      int64_t brows = b_h ? t.n : tm.k, bcols = b_h ? tm.k : t.n;
      if (tm.lda < acols || tm.a_off < 0 || tm.a_off + (arows - 1) * tm.lda + acols > a_len)
        return fail(CMPS_ERR_STATE, std::string(what) + ": A operand range outside its buffer");
      if (nsplit) {
        const int64_t bspan = (int64_t)((t.n - 1) / t.n_in) * tm.ldb_out + (t.n - 1) % t.n_in + 1;
        if (tm.ldb_out < t.n_in || tm.b_off < 0 || tm.b_off + (int64_t)(tm.k - 1) * tm.ldb + bspan > b_len)
          return fail(CMPS_ERR_STATE, std::string(what) + ": B operand range outside its buffer");
      } else if (tm.ldb < bcols || tm.b_off < 0 || tm.b_off + (brows - 1) * tm.ldb + bcols > b_len) {
        return fail(CMPS_ERR_STATE, std::string(what) + ": B operand range outside its buffer");
      }
    }
  }
  return CMPS_OK;
}

void GemmPlan::release() {
  if (d_tasks) dfree(d_tasks);
  if (d_terms) dfree(d_terms);
  if (d_tiles) dfree(d_tiles);
  d_tasks = nullptr;
  d_terms = nullptr;
  d_tiles = nullptr;
}


}  // namespace cmps
