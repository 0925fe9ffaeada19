// Split-precision (3-term TF32 or 3-term BF16 on tcgen05, FP32 accumulate)
// form of the H_eff matvec: operand preparation, tensor maps and the two
// stage plans.
//
// Layouts (split-TF32: FP32; S1A, LPS and RPTS as four planes re_hi, re_lo,
// im_hi, im_lo, TS as two planes re, im.  Split-BF16: 16-bit elements, every
// buffer -- TS included -- as four planes re_hi, re_mid, im_hi, im_mid):
//  * S1A  -- stage-1 A operand: theta transposed per (m, sigma1) chunk,
//            [r][a0] with r running over the padded right index of m (each
//            sigma2 chunk starts on a 4-element boundary) and ld = pad4(dim a0);
//  * LPS  -- stage-1 B operand: for every term of a (fused) task, the
//            LeftPart blocks [a0'][a0] of its column segments stacked along
//            a0', ld = pad4(dim a0);
//  * TS   -- stage-1 output = stage-2 A operand: T^{b1}_m as [l'][r_pad].
//            Split-TF32: the FP32 accumulator; stage 2 splits it into TF32
//            hi / lo in shared memory.  Split-BF16: the stage-1 epilogue
//            writes the four BF16 planes and stage 2 loads them by TMA.  Either
//            way T crosses HBM at 8 bytes per complex entry each way;
//  * RPTS -- stage-2 B operand: RightPart blocks transposed, [a2'][a2], the
//            blocks of a fused task's segments stacked along a2'.
// Every block base is 128-byte aligned and every leading dimension and K
// offset a multiple of 16 bytes (4 FP32, 8 BF16 elements), as the TMA
// requires; the K tail of every operand is zero-filled by the TMA
// (out-of-bounds fill), padding rows of S1A are zero.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>
#include <set>

#include "heff.h"
#include "split_common.cuh"
#include "tc_gemm.h"

namespace cmps {

struct SplitState {
  bool bf16 = false;                            // split-BF16 (16-bit elements) or split-TF32 (FP32)
  std::vector<int64_t> ldS;                     // per a0 sector
  std::vector<int64_t> ldR;                     // per a2 sector
  std::vector<std::vector<int64_t>> coloff_pad;  // [m][sigma2]
  std::vector<int64_t> ncols_pad;               // per m
  float* buf = nullptr;                         // one allocation for S1A, LPS, TS, RPTS (elements of 2 or 4 bytes)
  int64_t s1a_off = 0, s1a_len = 0, lps_off = 0, lps_len = 0, ts_off = 0, ts_len = 0, rpt_off = 0, rpt_len = 0;
  // theta -> S1A: one descriptor per (m, sigma1, sigma2) chunk, one per 32x32 tile
  void* d_theta_chunks = nullptr;
  void* d_theta_tiles = nullptr;
  int64_t n_theta_tiles = 0;
  int* d_err = nullptr;
  int* h_err = nullptr;  // pinned
  tc::TcPlan p1, p2;
  // element `off` of the buffer, as a raw pointer of the element type
  void* at(int64_t off) const { return bf16 ? (void*)((uint16_t*)buf + off) : (void*)(buf + off); }
  float* f32(int64_t off) const { return (float*)at(off); }
  int64_t pad(int64_t x) const { return bf16 ? (x + 7) & ~int64_t(7) : (x + 3) & ~int64_t(3); }
  int64_t align(int64_t x) const { return bf16 ? (x + 63) & ~int64_t(63) : (x + 31) & ~int64_t(31); }
};

namespace {

// A (m, sigma1, sigma2) chunk of theta: rows a0 (sector dim), columns a2,
// row-major inside its sector block; its S1A image is the transpose [a2][a0].
struct ThetaChunk {
  int64_t src_off, src_ld, dst_off, dst_ld;
  int32_t rows, cols;
};
struct ThetaTile {
  int32_t chunk, r0, c0, pad;
};

// theta -> split S1A, one 32 x 32 tile per CTA, transposed through shared
// memory so that both the FP64 reads and the plane writes coalesce.
template <class E>
struct Quad {
  E x, y, z, w;
};
template <class E>
__global__ void __launch_bounds__(256) k_split_theta_t(const ThetaTile* __restrict__ tiles,
                                                       const ThetaChunk* __restrict__ chunks,
                                                       const double* __restrict__ re, const double* __restrict__ im,
                                                       E* __restrict__ dst, int64_t plane) {
  __shared__ Quad<E> t[32][33];
  const ThetaTile tl = tiles[blockIdx.x];
  const ThetaChunk c = chunks[tl.chunk];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int r = tl.r0 + ty + 8 * k, col = tl.c0 + tx;
    if (r < c.rows && col < c.cols) {
      const int64_t o = c.src_off + (int64_t)r * c.src_ld + col;
      Quad<E> v;
      split4(re[o], im[o], &v.x, &v.y, &v.z, &v.w);
      t[ty + 8 * k][tx] = v;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int col = tl.c0 + ty + 8 * k, r = tl.r0 + tx;
    if (r < c.rows && col < c.cols) {
      const Quad<E> v = t[tx][ty + 8 * k];
      const int64_t o = c.dst_off + (int64_t)col * c.dst_ld + r;
      dst[o] = v.x;
      dst[o + plane] = v.y;
      dst[o + 2 * plane] = v.z;
      dst[o + 3 * plane] = v.w;
    }
  }
}

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

}  // namespace

static int encoder() {
  if (g_encode) return CMPS_OK;
  cudaDriverEntryPointQueryResult q;
  void* fn = nullptr;
  CMPS_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
  if (q != cudaDriverEntryPointSuccess || !fn) return fail(CMPS_ERR_CUDA, "cuTensorMapEncodeTiled not available");
  g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  return CMPS_OK;
}

namespace tc {
// 3-D map over one operand block of 2- or 4-byte elements: (K, rows, 4
// planes); box (64 bytes of K, box_rows, 4).  `base` is the block's first
// element in plane 0, the planes lie `plane` elements apart, and the block
// (rows x ld, K used per row) must fit inside `room` elements from base.
int encode_map(bool bf16, const void* base, int64_t K, int64_t rows, int64_t ld, int64_t plane, int64_t room,
               int box_rows, CUtensorMap* out) {
  CMPS_TRY(encoder());
  const int64_t es_b = bf16 ? 2 : 4;
  if (((uintptr_t)base & 15) || (ld * es_b) % 16 || (plane * es_b) % 16 || K < 1 || rows < 1 || K > ld)
    return fail(CMPS_ERR_STATE, "tensor map: misaligned operand block");
  if ((rows - 1) * ld + K > room) return fail(CMPS_ERR_STATE, "tensor map: operand block outside its buffer");
  cuuint64_t dims[3] = {(cuuint64_t)K, (cuuint64_t)rows, 4};
  cuuint64_t strides[2] = {(cuuint64_t)(ld * es_b), (cuuint64_t)(plane * es_b)};
  if (box_rows < 16 || box_rows > 128 || (box_rows & 15)) return fail(CMPS_ERR_STATE, "tensor map: bad box height");
  cuuint32_t box[3] = {(cuuint32_t)(64 / es_b), (cuuint32_t)box_rows, 4};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = g_encode(out, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                        const_cast<void*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(CMPS_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return CMPS_OK;
}
}  // namespace tc

namespace {

// A map over block `base_off` of a role of the split buffer (planes `plane`
// elements apart from element role_off); the block must lie inside the plane.
int make_map(const SplitState& S, int64_t role_off, int64_t base_off, int64_t K, int64_t rows, int64_t ld,
             int64_t plane, CUtensorMap* out, int box_rows = 128) {
  if (base_off < 0) return fail(CMPS_ERR_STATE, "tensor map: operand block outside its buffer");
  return tc::encode_map(S.bf16, S.at(role_off + base_off), K, rows, ld, plane, plane - base_off, box_rows, out);
}

}  // namespace

namespace tc {
void add_tiles(TcPlan& p, int32_t task, int32_t m, int32_t n) {
  for (int32_t m0 = 0; m0 < m; m0 += 128)
    for (int32_t n0 = 0; n0 < n; n0 += 128)
      p.tiles.push_back(TcTile{task, m0, n0, b_box_rows(n), 0, ((std::min(128, n - n0)) + 15) & ~15});
}

void mark_vector_stores(TcPlan& p, const void* out, int64_t plane) {
  for (TcTask& t : p.tasks) {
    bool ok = ((uintptr_t)out & 15) == 0 && t.row_stride == 1 && t.m % 8 == 0 && t.col_stride % 8 == 0 &&
              plane % 8 == 0 && t.nseg >= 1 && t.nseg <= 4;
    for (int q = 0; q < t.nseg && ok; ++q) ok = t.seg_off[q] >= 0 && t.seg_off[q] % 8 == 0;
    t.vstore = ok ? 1 : 0;
  }
}

int finish_plan(TcPlan& p, bool bf16, bool by_tma, const std::vector<int32_t>& b_rows, bool heaviest_first,
                bool wide_ok) {
  for (const TcTask& t : p.tasks)
    if (t.vstore && (t.row_stride != 1 || t.m % 8 || t.col_stride % 8))
      return fail(CMPS_ERR_STATE, "tcgen05 plan: vector stores on an unsuitable output");
  // k-steps per tile (the MMA warp walks them without term lookups)
  const int32_t ks = kstep(bf16);
  for (TcTile& t : p.tiles) {
    if (t.task < 0 || t.task >= (int32_t)p.tasks.size()) return fail(CMPS_ERR_STATE, "tcgen05 plan: bad tile");
    const TcTask& k = p.tasks[t.task];
    if (k.t0 < 0 || k.t1 < k.t0 || k.t1 > (int32_t)p.terms.size()) return fail(CMPS_ERR_STATE, "tcgen05 plan: bad task");
    int64_t it = 0;
    for (int q = k.t0; q < k.t1; ++q) it += (p.terms[q].k + ks - 1) / ks;
    if (it > 0x7fffffff) return fail(CMPS_ERR_ARG, "tcgen05 plan: too many k-steps in one tile");
    t.kiters = (int32_t)it;
    t.wide = wide_ok && bf16 && t.nmma <= 32 && t.b_rows == t.nmma ? 1 : 0;
  }
  // heaviest tiles first: the persistent kernel deals tiles round-robin to
  // the SMs, so this ordering balances the per-SM work
  if (heaviest_first) {
    auto cost = [&](const TcTile& t) {
      return (int64_t)(t.kiters + 2) * (t.nmma / 16);  // +2: fixed per-tile cost (epilogue)
    };
    std::stable_sort(p.tiles.begin(), p.tiles.end(), [&](const TcTile& a, const TcTile& b) { return cost(a) > cost(b); });
  }
  // plan integrity: every term names an existing map, every tile an existing task
  const int32_t na = (int32_t)(by_tma ? p.amaps.size() : p.adescs.size());
  // a TMA copy starts on a 16-byte boundary: the K offset a multiple of
  // 4 FP32 or 8 BF16 elements; a row offset only for A tiles loaded by TMA
  const int32_t amask = bf16 ? 7 : 3;
  for (const TcTerm& tm : p.terms)
    if (tm.a_map < 0 || tm.a_map >= na || tm.b_map < 0 || tm.b_map >= (int32_t)p.bmaps.size() || tm.k < 1 ||
        (tm.a_x0 & amask) || tm.a_y0 < 0 || (!by_tma && tm.a_y0 != 0))
      return fail(CMPS_ERR_STATE, "tcgen05 plan: bad term");
  for (const TcTask& t : p.tasks)
    if (t.t0 < 0 || t.t1 < t.t0 || t.t1 > (int32_t)p.terms.size() || t.m < 1 || t.n < 1 || t.out_off < 0)
      return fail(CMPS_ERR_STATE, "tcgen05 plan: bad task");
  // segments: start at column 0, increase, cover N; a task wider than one
  // 128-column tile has a single segment
  for (const TcTask& t : p.tasks) {
    if (t.nseg < 1 || t.nseg > 4 || t.seg_n0[0] != 0 || t.seg_off[0] != t.out_off || (t.nseg > 1 && t.n > 128))
      return fail(CMPS_ERR_STATE, "tcgen05 plan: bad segments");
    for (int q = 1; q < 4; ++q) {
      if (q < t.nseg ? (t.seg_n0[q] <= t.seg_n0[q - 1] || t.seg_n0[q] >= t.n || t.seg_off[q] < 0)
                     : t.seg_n0[q] != 0x7fffffff)
        return fail(CMPS_ERR_STATE, "tcgen05 plan: bad segments");
    }
  }
  // every B map of a task has the task's N rows, so the tile's B box height
  // (and the transaction bytes the producer expects) matches each map
  if (b_rows.size() != p.bmaps.size()) return fail(CMPS_ERR_STATE, "tcgen05 plan: B map count");
  for (const TcTask& t : p.tasks)
    for (int q = t.t0; q < t.t1; ++q)
      if (b_rows[p.terms[q].b_map] != t.n) return fail(CMPS_ERR_STATE, "tcgen05 plan: B map rows differ from N");
  for (const TcTile& tl : p.tiles) {
    const TcTask& t = p.tasks[tl.task];
    if (tl.m0 < 0 || tl.m0 >= t.m || tl.n0 < 0 || tl.n0 >= t.n) return fail(CMPS_ERR_STATE, "tcgen05 plan: tile origin");
    if (tl.b_rows != b_box_rows(t.n)) return fail(CMPS_ERR_STATE, "tcgen05 plan: B box height");
    if (tl.nmma < 16 || tl.nmma > 128 || tl.nmma != ((std::min(128, t.n - tl.n0) + 15) & ~15) || tl.nmma > tl.b_rows)
      return fail(CMPS_ERR_STATE, "tcgen05 plan: tile N");
  }
  return CMPS_OK;
}

int TcPlan::upload(cudaStream_t st) {
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
  CMPS_TRY(up(amaps, &d_amaps));
  CMPS_TRY(up(bmaps, &d_bmaps));
  CMPS_TRY(up(adescs, &d_adescs));
  return CMPS_OK;
}
void TcPlan::release() {
  if (d_adescs) dfree(d_adescs);
  d_adescs = nullptr;
  if (d_tasks) dfree(d_tasks);
  if (d_terms) dfree(d_terms);
  if (d_tiles) dfree(d_tiles);
  if (d_amaps) dfree(d_amaps);
  if (d_bmaps) dfree(d_bmaps);
  d_tasks = nullptr;
  d_terms = nullptr;
  d_tiles = nullptr;
  d_amaps = nullptr;
  d_bmaps = nullptr;
}
}  // namespace tc

void release_split(Heff* h) {
  if (h) h->low_canonical = false;  // the FP32 canonical operands go with the canonical plans
  release_canonical_tc(h);
  if (!h || !h->split) return;
  SplitState* s = h->split;
  s->p1.release();
  s->p2.release();
  if (s->buf) dfree(s->buf);
  if (s->d_theta_chunks) dfree(s->d_theta_chunks);
  if (s->d_theta_tiles) dfree(s->d_theta_tiles);
  if (s->d_err) dfree(s->d_err);
  if (s->h_err) cudaFreeHost(s->h_err);
  delete s;
  h->split = nullptr;
}

#ifndef CMPS_FUSE_MAX_SEG_N1
#define CMPS_FUSE_MAX_SEG_N1 64
#endif
#ifndef CMPS_FUSE_MAX_SEG_N2
#define CMPS_FUSE_MAX_SEG_N2 64
#endif
// widest task (column count) that is fused with others along N, per stage
constexpr int32_t kFuseMaxSegN1 = CMPS_FUSE_MAX_SEG_N1;
constexpr int32_t kFuseMaxSegN2 = CMPS_FUSE_MAX_SEG_N2;

static int build_split(Heff& H, bool bf16) {
  const Rules& r = H.rules;
  const ThetaSpace& th = H.th;
  const Bond& A0 = H.L.a;
  const Bond& A2 = H.R.a;
  const int d = H.d, nm = (int)th.mq.size();
  auto* S = new SplitState();
  H.split = S;
  S->bf16 = bf16;
  S->ldS.resize(A0.nsec());
  for (int s = 0; s < A0.nsec(); ++s) S->ldS[s] = S->pad(A0.sdim[s]);
  S->ldR.resize(A2.nsec());
  for (int t = 0; t < A2.nsec(); ++t) S->ldR[t] = S->pad(A2.sdim[t]);
  S->coloff_pad.assign(nm, std::vector<int64_t>(d, -1));
  S->ncols_pad.assign(nm, 0);
  for (int m = 0; m < nm; ++m) {
    int64_t o = 0;
    for (int s2 = 0; s2 < d; ++s2) {
      if (th.coloff[m][s2] < 0) continue;
      int t = A2.find(r.add(th.mq[m], H.sigq[s2]));
      S->coloff_pad[m][s2] = o;
      o += S->pad(A2.sdim[t]);
    }
    S->ncols_pad[m] = o;
  }
  // ---- sizes and offsets (elements per plane) ----
  std::map<std::pair<int, int>, int64_t> s1a_chunk;  // (m, sigma1) -> offset
  int64_t s1a = 0;
  for (int m = 0; m < nm; ++m)
    for (int s1 = 0; s1 < d; ++s1) {
      if (th.rowoff[m][s1] < 0) continue;
      int s = A0.find(r.sub(th.mq[m], H.sigq[s1]));
      s1a_chunk[{m, s1}] = s1a;
      s1a += S->align(S->ncols_pad[m] * S->ldS[s]);
    }
  std::vector<int64_t> ts_base((size_t)H.D * nm, -1);
  int64_t ts = 0;
  for (int b1 = 0; b1 < H.D; ++b1)
    for (int m = 0; m < nm; ++m) {
      if (H.t_base[(size_t)b1 * nm + m] < 0) continue;
      int mp = th.find(r.add(th.mq[m], H.bq[b1]));
      ts_base[(size_t)b1 * nm + m] = ts;
      ts += S->align(th.nrows[mp] * S->ncols_pad[m]);
    }
  // ---- tasks, fused along N ----
  // A stage-1 task (b1, sigma1') computes rows sigma1' of T^{b1}_m; a stage-2
  // task (m', sigma2') columns sigma2' of theta'_m'.  Tasks of one stage whose
  // term lists read the same A tiles (stage 1: the same m and sigma1 list;
  // stage 2: the same m' and (b1, sigma2) list) are fused into one task of up
  // to four column segments and N <= 128: the A tiles, the larger operand for
  // narrow sectors, are then loaded once for all of them.  Each fused term's
  // B rows are laid out contiguously (one tensor map per fused term), and the
  // epilogue sends each column to its segment's output.
  struct Seg {
    int64_t out_off;
    int32_t n;
    std::vector<std::array<int, 4>> keys;  // LP / RP block of every term
  };
  struct Fused {
    int m = 0;                             // stage 1: m; stage 2: m'
    int32_t ntot = 0;
    std::vector<std::array<int, 4>> tk;    // stage 1: (s1, s, 0, 0); stage 2: (b1, m, s2, t)
    std::vector<Seg> segs;
  };
  auto fuse = [](std::vector<std::pair<std::vector<int64_t>, std::pair<Fused, Seg>>>& raw, int32_t max_seg_n) {
    // raw: (signature, (task shape, its segment)) in creation order
    std::map<std::vector<int64_t>, std::vector<size_t>> groups;
    std::vector<std::vector<int64_t>> order;
    for (size_t i = 0; i < raw.size(); ++i) {
      auto it = groups.find(raw[i].first);
      if (it == groups.end()) {
        order.push_back(raw[i].first);
        groups[raw[i].first].push_back(i);
      } else {
        it->second.push_back(i);
      }
    }
    std::vector<Fused> out;
    for (const auto& sig : order) {
      Fused cur;
      bool open = false;
      for (size_t i : groups[sig]) {
        Seg& sg = raw[i].second.second;
        const bool fits = open && sg.n <= max_seg_n && cur.ntot + sg.n <= 128 && cur.segs.size() < 4 &&
                          cur.segs[0].n <= max_seg_n;
        if (!fits) {
          if (open) out.push_back(std::move(cur));
          cur = raw[i].second.first;
          cur.ntot = 0;
          cur.segs.clear();
          open = true;
        }
        cur.ntot += sg.n;
        cur.segs.push_back(std::move(sg));
      }
      if (open) out.push_back(std::move(cur));
    }
    return out;
  };
  std::vector<Fused> f1, f2;
  {
    std::vector<std::pair<std::vector<int64_t>, std::pair<Fused, Seg>>> raw;
    for (int b1 = 0; b1 < H.D; ++b1)
      for (int m = 0; m < nm; ++m) {
        const int64_t tb = ts_base[(size_t)b1 * nm + m];
        if (tb < 0) continue;
        const int mp = th.find(r.add(th.mq[m], H.bq[b1]));
        for (int s1p = 0; s1p < d; ++s1p) {
          if (th.rowoff[mp][s1p] < 0) continue;
          const int sp = A0.find(r.sub(th.mq[mp], H.sigq[s1p]));
          Fused shape;
          shape.m = m;
          Seg sg{tb + th.rowoff[mp][s1p] * S->ncols_pad[m], (int32_t)A0.sdim[sp], {}};
          std::vector<int64_t> sig{(int64_t)m};
          for (int s1 = 0; s1 < d; ++s1) {
            if (th.rowoff[m][s1] < 0) continue;
            const int sa = A0.find(r.sub(th.mq[m], H.sigq[s1]));
            if (!H.lp_off.count({b1, s1p, s1, sa})) continue;
            shape.tk.push_back({s1, sa, 0, 0});
            sg.keys.push_back({b1, s1p, s1, sa});
            sig.push_back(s1);
          }
          raw.push_back({sig, {shape, sg}});
        }
      }
    f1 = fuse(raw, kFuseMaxSegN1);
  }
  {
    std::vector<std::pair<std::vector<int64_t>, std::pair<Fused, Seg>>> raw;
    for (int mp = 0; mp < nm; ++mp)
      for (int s2p = 0; s2p < d; ++s2p) {
        if (th.coloff[mp][s2p] < 0 || !H.owned[mp]) continue;  // output sectors of this shard only
        const int tp = A2.find(r.add(th.mq[mp], H.sigq[s2p]));
        Fused shape;
        shape.m = mp;
        if (H.out_base[mp] < 0) return fail(CMPS_ERR_ARG, "output window lacks an owned sector");
        Seg sg{H.out_base[mp] + th.coloff[mp][s2p], (int32_t)A2.sdim[tp], {}};
        std::vector<int64_t> sig{(int64_t)mp};
        for (int b1 = 0; b1 < H.D; ++b1) {
          const int m = th.find(r.sub(th.mq[mp], H.bq[b1]));
          if (m < 0 || ts_base[(size_t)b1 * nm + m] < 0) continue;
          for (int s2 = 0; s2 < d; ++s2) {
            if (th.coloff[m][s2] < 0) continue;
            const int t = A2.find(r.add(th.mq[m], H.sigq[s2]));
            if (!H.rp_off.count({b1, s2, s2p, t})) continue;
            shape.tk.push_back({b1, m, s2, t});
            sg.keys.push_back({b1, s2, s2p, t});
            sig.push_back((int64_t)b1 * 65536 + s2);
          }
        }
        raw.push_back({sig, {shape, sg}});
      }
    f2 = fuse(raw, kFuseMaxSegN2);
  }
  // LPS / RPTS: one block per fused term, rows = the fused N (segment rows in
  // order), ld = pad4(K); every LP / RP block is split into its segment's rows
  std::vector<SplitBlock> lpsb, rptb;
  std::vector<std::vector<int64_t>> f1_base(f1.size()), f2_base(f2.size());
  int64_t lps = 0, rpt = 0;
  for (size_t i = 0; i < f1.size(); ++i) {
    const Fused& f = f1[i];
    for (size_t q = 0; q < f.tk.size(); ++q) {
      const int sa = f.tk[q][1];
      const int64_t ld = S->ldS[sa];
      f1_base[i].push_back(lps);
      int64_t row = 0;
      for (const Seg& sg : f.segs) {
        lpsb.push_back(SplitBlock{H.lp_off.at(sg.keys[q]), lps + row * ld, sg.n, (int32_t)A0.sdim[sa], (int32_t)ld, 0});
        row += sg.n;
      }
      lps += S->align(f.ntot * ld);
    }
  }
  for (size_t i = 0; i < f2.size(); ++i) {
    const Fused& f = f2[i];
    for (size_t q = 0; q < f.tk.size(); ++q) {
      const int t = f.tk[q][3];
      const int64_t ld = S->ldR[t];
      f2_base[i].push_back(rpt);
      int64_t row = 0;
      for (const Seg& sg : f.segs) {
        // RP block is [a2][a2'] (dim t x dim t'); stored transposed [a2'][a2]
        rptb.push_back(SplitBlock{H.rp_off.at(sg.keys[q]), rpt + row * ld, (int32_t)A2.sdim[t], sg.n, (int32_t)ld, 1});
        row += sg.n;
      }
      rpt += S->align(f.ntot * ld);
    }
  }
  S->s1a_off = 0;
  S->s1a_len = S->align(std::max<int64_t>(s1a, 32));
  S->lps_off = 4 * S->s1a_len;
  S->lps_len = S->align(std::max<int64_t>(lps, 32));
  S->ts_off = S->lps_off + 4 * S->lps_len;
  S->ts_len = S->align(std::max<int64_t>(ts, 32));
  S->rpt_off = S->ts_off + (S->bf16 ? 4 : 2) * S->ts_len;  // T: two FP32 planes (re, im) or four BF16
  S->rpt_len = S->align(std::max<int64_t>(rpt, 32));
  const int64_t total = S->rpt_off + 4 * S->rpt_len;
  const size_t ebytes = S->bf16 ? 2 : 4;
  if (dmalloc(&S->buf, ebytes * total) != cudaSuccess)
    return fail(CMPS_ERR_NOMEM, "split-TF32 operand allocation failed");
  // zero fill: padding rows and columns of every operand must read as zero
  CMPS_TRY(zero_wait(S->buf, ebytes * total, H.ctx->stream));
  CMPS_CUDA(dmalloc(&S->d_err, sizeof(int)));
  CMPS_TRY(zero_wait(S->d_err, sizeof(int), H.ctx->stream));
  CMPS_CUDA(cudaMallocHost(&S->h_err, sizeof(int)));
  // ---- split LeftPart / RightPart ----
  {
    SplitBlock* d = nullptr;
    for (int pass = 0; pass < 2; ++pass) {
      std::vector<SplitBlock>& v = pass == 0 ? lpsb : rptb;
      if (v.empty()) continue;
      for (auto& b : v) {
        const int64_t rows = b.transpose ? b.cols : b.rows;  // rows of the destination layout
        const int64_t cols = b.transpose ? b.rows : b.cols;
        const int64_t len = pass == 0 ? S->lps_len : S->rpt_len;
        if (b.dst_off + (rows - 1) * b.ld_dst + cols > len || b.ld_dst < cols)
          return fail(CMPS_ERR_STATE, "split block outside its buffer");
      }
      CMPS_CUDA(dmalloc(&d, sizeof(SplitBlock) * v.size()));
      CMPS_TRY(copy_wait(d, v.data(), sizeof(SplitBlock) * v.size(), cudaMemcpyHostToDevice, H.ctx->stream));
      const Planar& src = pass == 0 ? H.LP : H.RP;
      const int64_t plane = pass == 0 ? S->lps_len : S->rpt_len;
      void* dst = S->at(pass == 0 ? S->lps_off : S->rpt_off);
      if (S->bf16)
        k_split_blocks<uint16_t><<<(unsigned)v.size(), 256, 0, H.ctx->stream>>>(d, src.re(), src.im(),
                                                                               (uint16_t*)dst, plane);
      else
        k_split_blocks<float><<<(unsigned)v.size(), 256, 0, H.ctx->stream>>>(d, src.re(), src.im(), (float*)dst,
                                                                            plane);
      CMPS_CUDA(cudaGetLastError());
      CMPS_CUDA(cudaStreamSynchronize(H.ctx->stream));
      dfree(d);
    }
  }
  // ---- theta -> S1A chunk and tile descriptors ----
  {
    std::vector<ThetaChunk> chunks;
    std::vector<ThetaTile> tiles;
    for (int m = 0; m < nm; ++m)
      for (int s1 = 0; s1 < d; ++s1) {
        if (th.rowoff[m][s1] < 0 || !H.in_need[m]) continue;  // only the sectors the owned outputs read
        if (H.in_base[m] < 0) return fail(CMPS_ERR_ARG, "input window lacks a sector the owned outputs read");
        int s = A0.find(r.sub(th.mq[m], H.sigq[s1]));
        const int64_t ch = s1a_chunk[{m, s1}];
        for (int s2 = 0; s2 < d; ++s2) {
          if (th.coloff[m][s2] < 0) continue;
          int t = A2.find(r.add(th.mq[m], H.sigq[s2]));
          ThetaChunk c{};
          c.src_off = H.in_base[m] + th.rowoff[m][s1] * th.ncols[m] + th.coloff[m][s2];
          c.src_ld = th.ncols[m];
          c.dst_off = ch + S->coloff_pad[m][s2] * S->ldS[s];
          c.dst_ld = S->ldS[s];
          c.rows = (int32_t)A0.sdim[s];
          c.cols = (int32_t)A2.sdim[t];
          // both images inside their buffers
          if (c.src_off + (int64_t)(c.rows - 1) * c.src_ld + c.cols > H.in_len ||
              c.dst_off + (int64_t)(c.cols - 1) * c.dst_ld + c.rows > S->s1a_len || c.dst_ld < c.rows)
            return fail(CMPS_ERR_STATE, "theta split chunk outside its buffer");
          for (int32_t r0 = 0; r0 < c.rows; r0 += 32)
            for (int32_t c0 = 0; c0 < c.cols; c0 += 32) tiles.push_back(ThetaTile{(int32_t)chunks.size(), r0, c0, 0});
          chunks.push_back(c);
        }
      }
    if (tiles.size() > 0x7fffffffull) return fail(CMPS_ERR_ARG, "too many theta tiles");
    S->n_theta_tiles = (int64_t)tiles.size();
    if (!chunks.empty()) {
      CMPS_CUDA(dmalloc(&S->d_theta_chunks, sizeof(ThetaChunk) * chunks.size()));
      CMPS_TRY(copy_wait(S->d_theta_chunks, chunks.data(), sizeof(ThetaChunk) * chunks.size(), cudaMemcpyHostToDevice,
                         H.ctx->stream));
      CMPS_CUDA(dmalloc(&S->d_theta_tiles, sizeof(ThetaTile) * tiles.size()));
      CMPS_TRY(copy_wait(S->d_theta_tiles, tiles.data(), sizeof(ThetaTile) * tiles.size(), cudaMemcpyHostToDevice,
                         H.ctx->stream));
    }
  }
  // ---- stage 1 plan: C1[r_pad, a0'] = sum S1A[r_pad, a0] LPS[a0', a0] ----
  tc::TcPlan& p1 = S->p1;
  std::map<std::pair<int, int>, int32_t> amap1;
  for (auto& kv : s1a_chunk) {
    int m = kv.first.first, s1 = kv.first.second;
    int s = A0.find(r.sub(th.mq[m], H.sigq[s1]));
    CUtensorMap cm;
    CMPS_TRY(make_map(*S, S->s1a_off, kv.second, A0.sdim[s], S->ncols_pad[m], S->ldS[s], S->s1a_len, &cm));
    amap1[kv.first] = (int32_t)p1.amaps.size();
    p1.amaps.push_back(cm);
  }
  std::vector<int32_t> b1_rows, b2_rows;  // row extent of every B map (= its task's N)
  auto set_segments = [](tc::TcTask& task, const std::vector<Seg>& segs) {
    task.nseg = (int32_t)segs.size();
    int32_t col = 0;
    for (int q = 0; q < 4; ++q) {
      task.seg_n0[q] = q < (int)segs.size() ? col : 0x7fffffff;
      task.seg_off[q] = q < (int)segs.size() ? segs[q].out_off : 0;
      if (q < (int)segs.size()) col += segs[q].n;
    }
    task.out_off = segs[0].out_off;
  };
  for (size_t i = 0; i < f1.size(); ++i) {
    const Fused& f = f1[i];
    const int m = f.m;
    tc::TcTask task{};
    set_segments(task, f.segs);
    task.row_stride = 1;
    task.col_stride = S->ncols_pad[m];
    task.m = (int32_t)S->ncols_pad[m];
    task.n = f.ntot;
    task.t0 = (int32_t)p1.terms.size();
    for (size_t q = 0; q < f.tk.size(); ++q) {
      const int s1 = f.tk[q][0], sa = f.tk[q][1];
      CUtensorMap cm;
      CMPS_TRY(make_map(*S, S->lps_off, f1_base[i][q], A0.sdim[sa], f.ntot, S->ldS[sa], S->lps_len, &cm,
                        tc::b_box_rows(f.ntot)));
      p1.terms.push_back(tc::TcTerm{amap1[{m, s1}], (int32_t)p1.bmaps.size(), 0, (int32_t)A0.sdim[sa]});
      p1.bmaps.push_back(cm);
      b1_rows.push_back(f.ntot);
    }
    task.t1 = (int32_t)p1.terms.size();
    // output range check of every segment (two FP32 or four BF16 planes of TS)
    for (const Seg& sg : f.segs)
      if (sg.out_off < 0 || sg.out_off + (int64_t)(task.m - 1) * task.row_stride + (int64_t)(sg.n - 1) * task.col_stride >=
                                S->ts_len)
        return fail(CMPS_ERR_STATE, "stage-1 output outside TS");
    tc::add_tiles(p1, (int32_t)p1.tasks.size(), task.m, task.n);
    p1.tasks.push_back(task);
  }
  // ---- stage 2 plan: C2[l', a2'] = sum TS[l', r_pad] RPTS[a2', a2] ----
  tc::TcPlan& p2 = S->p2;
  std::vector<int32_t> amap2((size_t)H.D * nm, -1);
  for (int b1 = 0; b1 < H.D; ++b1)
    for (int m = 0; m < nm; ++m) {
      const int64_t tb = ts_base[(size_t)b1 * nm + m];
      if (tb < 0) continue;
      int mp = th.find(r.add(th.mq[m], H.bq[b1]));
      if (S->bf16) {
        // T^{b1}_m as four BF16 planes, loaded by TMA
        CUtensorMap cm;
        CMPS_TRY(make_map(*S, S->ts_off, tb, S->ncols_pad[m], th.nrows[mp], S->ncols_pad[m], S->ts_len, &cm));
        amap2[(size_t)b1 * nm + m] = (int32_t)p2.amaps.size();
        p2.amaps.push_back(cm);
        continue;
      }
      // T^{b1}_m as two FP32 planes, read and split by the converter warps
      tc::TcADesc ad{tb, S->ncols_pad[m], (int32_t)th.nrows[mp], (int32_t)S->ncols_pad[m]};
      if (tb < 0 || tb % 4 || ad.ld % 4 || tb + (ad.rows - 1) * ad.ld + ad.cols > S->ts_len)
        return fail(CMPS_ERR_STATE, "stage-2 A block outside T");
      amap2[(size_t)b1 * nm + m] = (int32_t)p2.adescs.size();
      p2.adescs.push_back(ad);
    }
  for (size_t i = 0; i < f2.size(); ++i) {
    const Fused& f = f2[i];
    const int mp = f.m;
    tc::TcTask task{};
    set_segments(task, f.segs);
    task.row_stride = th.ncols[mp];
    task.col_stride = 1;
    task.m = (int32_t)th.nrows[mp];
    task.n = f.ntot;
    task.t0 = (int32_t)p2.terms.size();
    for (size_t q = 0; q < f.tk.size(); ++q) {
      const int b1 = f.tk[q][0], m = f.tk[q][1], s2 = f.tk[q][2], t = f.tk[q][3];
      const int32_t am = amap2[(size_t)b1 * nm + m];
      if (am < 0) return fail(CMPS_ERR_STATE, "stage-2 term without its T block");
      CUtensorMap cm;
      // destination layout [a2'][a2]: rows = fused N, K = dim t
      CMPS_TRY(make_map(*S, S->rpt_off, f2_base[i][q], A2.sdim[t], f.ntot, S->ldR[t], S->rpt_len, &cm,
                        tc::b_box_rows(f.ntot)));
      p2.terms.push_back(tc::TcTerm{am, (int32_t)p2.bmaps.size(), (int32_t)S->coloff_pad[m][s2], (int32_t)A2.sdim[t]});
      p2.bmaps.push_back(cm);
      b2_rows.push_back(f.ntot);
    }
    task.t1 = (int32_t)p2.terms.size();
    for (const Seg& sg : f.segs)
      if (sg.out_off < 0 || sg.out_off + (int64_t)(task.m - 1) * task.row_stride + (int64_t)(sg.n - 1) * task.col_stride >=
                                H.out_len)
        return fail(CMPS_ERR_STATE, "stage-2 output outside theta");
    tc::add_tiles(p2, (int32_t)p2.tasks.size(), task.m, task.n);
    p2.tasks.push_back(task);
  }
  if (S->bf16) tc::mark_vector_stores(p1, S->at(S->ts_off), S->ts_len);
  CMPS_TRY(tc::finish_plan(p1, S->bf16, true, b1_rows, true));
  CMPS_TRY(tc::finish_plan(p2, S->bf16, S->bf16, b2_rows, true));
  if (!S->bf16)
    for (const tc::TcTerm& tm : p2.terms)
      if (tm.a_x0 + tm.k > p2.adescs[tm.a_map].cols) return fail(CMPS_ERR_STATE, "tcgen05 plan: term past its T block");
  CMPS_TRY(p1.upload(H.ctx->stream));
  CMPS_TRY(p2.upload(H.ctx->stream));
  return CMPS_OK;
}

// The split-precision operator of a handle: the folded order on tcgen05
// (this file), or -- when the canonical order is requested, or executes at
// most a quarter of the folded order's flops -- the canonical order: on
// tcgen05 in split BF16 (canonical_tc.cu), else in FP32 (canonical.cu).  The
// quarter weighs the folded form's large-K tensor-core GEMMs against the
// canonical form's short-K stages and three intermediates in HBM.
constexpr double kLowCanonicalRatio = 0.25;

int prepare_precision(Heff* h, int precision) {
  if (precision == CMPS_FP64) return CMPS_OK;
  if (!is_split(precision)) return fail(CMPS_ERR_ARG, "unknown precision");
  const bool bf16 = precision == CMPS_SPLIT_BF16;
  // a split operator of the other format is rebuilt
  if (h->split && h->split->bf16 != bf16) release_split(h);
  if (h->low_canonical && (h->ctc != nullptr) != (bf16 && h->whole())) release_split(h);
  if (h->split || h->low_canonical) return CMPS_OK;
  if (h->canon && (h->order_req == CMPS_ORDER_CANONICAL || h->flops_canon <= kLowCanonicalRatio * h->flops_folded)) {
    if (bf16 && h->whole()) {
      const int st = build_canonical_tc(*h);
      if (st == CMPS_OK) {
        h->low_canonical = true;
        return CMPS_OK;
      }
      release_canonical_tc(h);
      if (st != CMPS_ERR_NOMEM) return st;
      cudaGetLastError();  // no room for the BF16 intermediates: the FP32 form
    }
    CMPS_TRY(build_canonical32(*h));
    h->low_canonical = true;
    return CMPS_OK;
  }
  int st = build_split(*h, bf16);
  if (st != CMPS_OK) release_split(h);
  return st;
}

int split_form(const Heff& H) {
  if (H.precision == CMPS_FP64) return CMPS_FORM_NONE;
  if (H.low_canonical) return H.ctc ? CMPS_FORM_CANONICAL_TC : CMPS_FORM_CANONICAL_FP32;
  return H.split ? CMPS_FORM_FOLDED_TC : CMPS_FORM_NONE;
}

// stage 1 (T = LeftPart . theta) or stage 2 (theta' = T . RightPart) of a
// prepared split operator: tcgen05 modes 1 / 2 (TF32) or 3 / 4 (BF16)
static int launch_stage(const SplitState& S, int which, Planar& out, cudaStream_t st) {
  if (which == 1)
    return tc::launch(S.bf16 ? 3 : 1, S.p1, S.f32(S.ts_off), S.ts_len, nullptr, 0, nullptr, 0, S.d_err, st);
  if (S.bf16) return tc::launch(4, S.p2, nullptr, 0, out.re(), out.len, nullptr, 0, S.d_err, st);
  return tc::launch(2, S.p2, nullptr, 0, out.re(), out.len, S.f32(S.ts_off), S.ts_len, S.d_err, st);
}

static int split_theta(const SplitState& S, const Planar& in, cudaStream_t st) {
  if (S.n_theta_tiles == 0) return CMPS_OK;
  if (S.bf16)
    k_split_theta_t<uint16_t><<<(unsigned)S.n_theta_tiles, 256, 0, st>>>(
        (const ThetaTile*)S.d_theta_tiles, (const ThetaChunk*)S.d_theta_chunks, in.re(), in.im(),
        (uint16_t*)S.at(S.s1a_off), S.s1a_len);
  else
    k_split_theta_t<float><<<(unsigned)S.n_theta_tiles, 256, 0, st>>>(
        (const ThetaTile*)S.d_theta_tiles, (const ThetaChunk*)S.d_theta_chunks, in.re(), in.im(),
        S.f32(S.s1a_off), S.s1a_len);
  CMPS_CUDA(cudaGetLastError());
  return CMPS_OK;
}

// The error word of the handle's tcgen05 pipelines (device, pinned host);
// false for the FP32 canonical form, which has no pipeline waits.
static bool error_words(const Heff& H, int** d_err, int** h_err) {
  *d_err = *h_err = nullptr;
  if (H.low_canonical) {
    canonical_tc_error_words(H, d_err, h_err);
  } else if (H.split) {
    *d_err = H.split->d_err;
    *h_err = H.split->h_err;
  }
  return *d_err != nullptr;
}

int split_reset_error(Heff& H, cudaStream_t st) {
  int *d_err, *h_err;
  if (!error_words(H, &d_err, &h_err)) {
    if (H.low_canonical) return CMPS_OK;
    return fail(CMPS_ERR_STATE, "split-precision operands not prepared");
  }
  CMPS_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), st));
  return CMPS_OK;
}

int apply_split_async(Heff& H, const Planar& in, Planar& out, cudaStream_t st) {
  if (H.low_canonical) {
    if (H.ctc)
      CMPS_TRY(apply_canonical_tc(H, 0, in, out, st));
    else
      CMPS_TRY(apply_canonical32(H, 0, in, out, st));
    return H.add_projectors(in, out, st);
  }
  SplitState* S = H.split;
  if (!S) return fail(CMPS_ERR_STATE, "split-precision operands not prepared");
  CMPS_TRY(split_theta(*S, in, st));
  CMPS_TRY(launch_stage(*S, 1, out, st));
  CMPS_TRY(launch_stage(*S, 2, out, st));
  return H.add_projectors(in, out, st);
}

// theta-space matvec in split precision: FP64 planar in -> FP64 planar out.
int apply_split(Heff& H, const Planar& in, Planar& out, cudaStream_t st) {
  int *d_err, *h_err;
  if (!error_words(H, &d_err, &h_err)) return apply_split_async(H, in, out, st);
  CMPS_TRY(split_reset_error(H, st));
  CMPS_TRY(apply_split_async(H, in, out, st));
  CMPS_CUDA(cudaMemcpyAsync(h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  CMPS_CUDA(cudaStreamSynchronize(st));
  if (*h_err) return fail(CMPS_ERR_CUDA, "tcgen05 pipeline wait timed out (code " + std::to_string(*h_err) + ")");
  return CMPS_OK;
}

int apply_split_stage(Heff& H, int which, const Planar& in, Planar& out, cudaStream_t st) {
  if (H.low_canonical && !H.ctc) return apply_canonical32(H, which, in, out, st);
  if (which == 1) CMPS_TRY(split_reset_error(H, st));
  if (H.ctc) return apply_canonical_tc(H, which, in, out, st);
  SplitState* S = H.split;
  if (!S) return fail(CMPS_ERR_STATE, "split-precision operands not prepared");
  if (which == 1) {
    CMPS_TRY(split_theta(*S, in, st));
    return launch_stage(*S, 1, out, st);
  }
  return launch_stage(*S, 2, out, st);
}

int split_error(Heff& H) {
  int *d_err, *h_err;
  if (!error_words(H, &d_err, &h_err)) return CMPS_OK;
  int e = 0;
  CMPS_TRY(copy_wait(&e, d_err, sizeof(int), cudaMemcpyDeviceToHost, H.ctx->stream));
  if (e) return fail(CMPS_ERR_CUDA, "tcgen05 pipeline wait timed out (code " + std::to_string(e) + ")");
  return CMPS_OK;
}

}  // namespace cmps
