// The split-BF16 H_eff matvec in the canonical contraction order, on the
// tcgen05 tensor cores (the persistent split GEMM of tc_gemm.cu, modes 3
// and 4).  The same linear map as the canonical FP64 order (canonical.cu)
// and as the reference's LeftPart . V . RightPart (TwoVertexMPOMPSMultiply,
// DMRG_routines.cpp:898-945), contracted one index at a time from the right:
//
//   Z^{b2}  = Theta . R^{b2}                          (stage R:  contract a2)
//   Y^{b1}  = sum_{b2, s2} W[s2', b1, s2, b2] Z^{b2}   (stage W2: contract sigma2)
//   V^{b0}  = sum_{b1, s1} W[s1', b0, s1, b1] Y^{b1}   (stage W1: contract sigma1)
//   Theta'  = sum_{b0} L^{b0} . V^{b0}                 (stage L:  contract a0)
//
// Layout rule.  The kernel computes C[m, n] = sum_k A[m, k] B[n, k] with both
// operands K-contiguous and writes C with m contiguous (one TMEM lane per
// row, so a warp's stores coalesce).  A stage's output is the next stage's A
// operand as it stands when the index the next stage contracts is the
// output's fastest one: each stage removes the fastest index and prepends
// its new index as the slowest.  With theta stored as [a0][s1][s2][a2] the
// indices are contracted in the order a2, s2, s1, a0, and every
// intermediate is in place for the next stage:
//   Theta_in  [a0][s1][s2][a2]     per (m, class c1, class c2)
//   Z^{b2}    [a2'][a0][s1][s2]    per (b2, m, c1, c2)
//   Y^{b1}    [s2'][a2'][a0][s1]   per (b1, m, c1, c2')
//   V^{b0}    [s1'][s2'][a2'][a0]  per (b0, m'', c1', c2')
// Stage L writes Theta'_{m''}[(s1', a0')][(s2', a2')] itself in FP64, one
// task per s1': its rows (s2', a2') are a contiguous run of a block row and
// a0' is the block's row index.  Only the input is reordered, (s1, a0) ->
// (a0, s1) on the way into the BF16 planes.  An index about to be contracted
// is padded to a multiple of 8 (16-byte TMA rows); Theta_in's padding is
// zero, and no intermediate's padding is read (the tensor maps' K extents
// stop at the true dimension and the TMA fills the rest with zeros).
//
// Charges, additive: q(a0) + q(s1) = m = q(a2) - q(s2) for Theta_m.  R^{b2}
// takes the a2 sector t to R.partner(b2, t), L^{b0} the a0 sector s to
// L.partner(b0, s).  Z^{b2}_{m,c1,c2} therefore has a2' in
// R.partner(b2, sector(m + q(c2))); Y^{b1}_{m,c1,c2'} belongs to the output
// block m'' = m + q(b1) and has a2' in sector(m'' + q(c2')); V^{b0} has a0
// in the sector L^{b0} maps onto sector(m'' - q(c1')), the a0' of the
// output rows of class c1'.
//
// Every operand is split into BF16 planes re_hi, re_mid, im_hi, im_mid and
// accumulated in FP32 in TMEM (three products per real product); each
// intermediate is written already split, 8 bytes per complex entry.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <map>
#include <set>
#include <tuple>

#include "heff.h"
#include "split_common.cuh"
#include "tc_gemm.h"

namespace cmps {

namespace {

// One (m, c1, c2) block of theta on its way into Theta_in: theta_m rows
// rcoff + i * d0 + a0, columns ccoff + j * d2 + a2 (src = the in-plane offset
// of row rcoff, column ccoff; ncols the block's row length) to
// dst + ((a0 * n1p + i) * n2p + j) * d2p + a2.
struct XinBlock {
  int64_t src, ncols, dst;
  int32_t d0, n1, n2, d2;
  int32_t n1p, n2p, d2p, pad;
};

// theta (FP64 planes) -> Theta_in (four BF16 planes): one warp per run of d2
// consecutive elements, which are consecutive in both layouts.
__global__ void __launch_bounds__(256) k_gather_theta(const XinBlock* __restrict__ blocks,
                                                      const double* __restrict__ re, const double* __restrict__ im,
                                                      uint16_t* __restrict__ dst, int64_t plane) {
  const XinBlock b = blocks[blockIdx.y];
  const int64_t runs = (int64_t)b.d0 * b.n1 * b.n2;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t step = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp; r < runs; r += step) {
    const int64_t j = r % b.n2, t = r / b.n2;
    const int64_t i = t % b.n1, a0 = t / b.n1;
    const int64_t s = b.src + (i * b.d0 + a0) * b.ncols + j * b.d2;
    const int64_t d = b.dst + ((a0 * b.n1p + i) * b.n2p + j) * b.d2p;
    for (int a2 = lane; a2 < b.d2; a2 += 32) {
      uint16_t* o = dst + d + a2;
      split4(re[s + a2], im[s + a2], o, o + plane, o + 2 * plane, o + 3 * plane);
    }
  }
}

inline int64_t pad8(int64_t x) { return (x + 7) & ~int64_t(7); }
inline int64_t align64(int64_t x) { return (x + 63) & ~int64_t(63); }

using Key4 = std::array<int, 4>;

}  // namespace

struct CanonTc {
  // four BF16 planes each (plane stride *_len elements)
  uint16_t* ops = nullptr;  // B operands: R^T, L and W blocks
  uint16_t* xin = nullptr;  // Theta_in
  uint16_t* zv = nullptr;   // Z, then V (Z is dead once stage W2 has run)
  uint16_t* y = nullptr;    // Y
  int64_t ops_len = 0, xin_len = 0, zv_len = 0, y_len = 0;
  bool own_zv = false, own_y = false;  // else views into the FP64 canonical intermediates
  XinBlock* d_xin = nullptr;
  int n_xin = 0;
  int64_t max_runs = 0;
  tc::TcPlan pR, pW2, pW1, pL;
  int* d_err = nullptr;
  int* h_err = nullptr;  // pinned
  double flops = 0.0;    // executed (padded) complex flops per matvec
  ~CanonTc() {
    for (tc::TcPlan* p : {&pR, &pW2, &pW1, &pL}) p->release();
    if (ops) dfree(ops);
    if (xin) dfree(xin);
    if (zv && own_zv) dfree(zv);
    if (y && own_y) dfree(y);
    if (d_xin) dfree(d_xin);
    if (d_err) dfree(d_err);
    if (h_err) cudaFreeHost(h_err);
  }
};

void release_canonical_tc(Heff* h) {
  if (!h || !h->ctc) return;
  delete h->ctc;
  h->ctc = nullptr;
}

void canonical_tc_error_words(const Heff& H, int** d_err, int** h_err) {
  *d_err = H.ctc ? H.ctc->d_err : nullptr;
  *h_err = H.ctc ? H.ctc->h_err : nullptr;
}

int build_canonical_tc(Heff& H) {
  release_canonical_tc(&H);
  if (!H.whole()) return fail(CMPS_ERR_STATE, "canonical tcgen05 form: sharded or windowed matvec");
  const Planar* fp64_xz = nullptr;
  const Planar* fp64_y = nullptr;
  CMPS_TRY(canonical_scratch(H, &fp64_xz, &fp64_y));
  const Rules& r = H.rules;
  const ThetaSpace& th = H.th;
  const Bond& A0 = H.L.a;
  const Bond& A2 = H.R.a;
  const int nm = (int)th.mq.size();
  const int ncls = (int)H.cls_mem.size();
  const int ns0 = A0.nsec(), ns2 = A2.nsec();
  cudaStream_t st = H.ctx->stream;
  // ---- class geometry of every theta block ----
  std::vector<std::vector<int64_t>> rcoff(nm, std::vector<int64_t>(ncls, -1)), rcdim = rcoff, ccoff = rcoff,
                                                                              ccdim = rcoff;
  std::vector<std::vector<int>> rsec(nm, std::vector<int>(ncls, -1)), csec = rsec;  // a0 / a2 sector of the class
  for (int m = 0; m < nm; ++m)
    for (int c = 0; c < ncls; ++c) {
      const std::vector<int>& mem = H.cls_mem[c];
      const QKey qc = H.sigq[mem[0]];
      if (th.rowoff[m][mem[0]] >= 0) {
        rsec[m][c] = A0.find(r.sub(th.mq[m], qc));
        rcoff[m][c] = th.rowoff[m][mem[0]];
        rcdim[m][c] = A0.sdim[rsec[m][c]];
        for (size_t i = 0; i < mem.size(); ++i)
          if (th.rowoff[m][mem[i]] != rcoff[m][c] + (int64_t)i * rcdim[m][c])
            return fail(CMPS_ERR_STATE, "canonical order: class rows not equally strided");
      }
      if (th.coloff[m][mem[0]] >= 0) {
        csec[m][c] = A2.find(r.add(th.mq[m], qc));
        ccoff[m][c] = th.coloff[m][mem[0]];
        ccdim[m][c] = A2.sdim[csec[m][c]];
        for (size_t i = 0; i < mem.size(); ++i)
          if (th.coloff[m][mem[i]] != ccoff[m][c] + (int64_t)i * ccdim[m][c])
            return fail(CMPS_ERR_STATE, "canonical order: class columns not equally strided");
      }
    }
  auto ncl = [&](int c) { return (int64_t)H.cls_mem[c].size(); };
  // MPO class blocks (bl, br, class in, class out), dense [n_out][n_in]
  std::map<Key4, std::vector<std::pair<int64_t, std::pair<double, double>>>> wblk;
  for (const WEntry& w : H.W) {
    const int ci = H.cls_of[w.s], co = H.cls_of[w.sp];
    wblk[{w.bl, w.br, ci, co}].push_back({(int64_t)H.cls_pos[w.sp] * ncl(ci) + H.cls_pos[w.s], {w.wr, w.wi}});
  }
  // by right bond: (br) -> blocks
  std::map<int, std::vector<Key4>> w_by_br;
  for (auto& kv : wblk) w_by_br[kv.first[1]].push_back(kv.first);

  // ---- what is needed, from the outputs backwards ----
  // V (b0, m'', c1', c2'): the a0 sector L^{b0} maps onto the output rows' a0'
  struct VKey {
    int b0, mpp, c1p, c2p;
    bool operator<(const VKey& o) const {
      return std::tie(b0, mpp, c1p, c2p) < std::tie(o.b0, o.mpp, o.c1p, o.c2p);
    }
  };
  std::map<VKey, int> v_alpha;
  for (int mpp = 0; mpp < nm; ++mpp)
    for (int c1p = 0; c1p < ncls; ++c1p) {
      if (rcoff[mpp][c1p] < 0) continue;
      const int a0p = rsec[mpp][c1p];
      for (int c2p = 0; c2p < ncls; ++c2p) {
        if (ccoff[mpp][c2p] < 0) continue;
        for (int b0 = 0; b0 < H.D; ++b0) {
          int alpha = -1;
          for (int s = 0; s < ns0; ++s)
            if (H.L.off[(size_t)b0 * ns0 + s] >= 0 && H.L.partner[(size_t)b0 * ns0 + s] == a0p) alpha = s;
          if (alpha >= 0) v_alpha[{b0, mpp, c1p, c2p}] = alpha;
        }
      }
    }
  // Y (b1, m, c1, c2') read by some V
  std::set<Key4> ycand;
  for (auto& kv : v_alpha) {
    const VKey& v = kv.first;
    for (auto& wk : wblk) {
      if (wk.first[0] != v.b0 || wk.first[3] != v.c1p) continue;
      const int b1 = wk.first[1], c1 = wk.first[2];
      const int m = th.find(r.sub(th.mq[v.mpp], H.bq[b1]));
      if (m < 0 || rcoff[m][c1] < 0) continue;
      if (rsec[m][c1] != kv.second) return fail(CMPS_ERR_STATE, "canonical tcgen05 form: W1 sector mismatch");
      ycand.insert({b1, m, c1, v.c2p});
    }
  }
  // Z (b2, m, c1, c2) read by some Y
  std::set<Key4> zset;
  for (const Key4& yk : ycand) {
    const int b1 = yk[0], m = yk[1], c1 = yk[2], c2p = yk[3];
    const int mpp = th.find(r.add(th.mq[m], H.bq[b1]));
    if (mpp < 0 || ccoff[mpp][c2p] < 0) continue;
    for (auto& wk : wblk) {
      if (wk.first[0] != b1 || wk.first[3] != c2p) continue;
      const int b2 = wk.first[1], c2 = wk.first[2];
      if (ccoff[m][c2] < 0) continue;
      const int t = csec[m][c2];
      if (H.R.off[(size_t)b2 * ns2 + t] < 0) continue;
      if (H.R.partner[(size_t)b2 * ns2 + t] != csec[mpp][c2p])
        return fail(CMPS_ERR_STATE, "canonical tcgen05 form: W2 sector mismatch");
      zset.insert({b2, m, c1, c2});
    }
  }

  auto* T = new (std::nothrow) CanonTc();
  if (!T) return fail(CMPS_ERR_NOMEM, "host allocation failed");
  H.ctc = T;
  // ---- Theta_in blocks ----
  std::map<std::array<int, 3>, int64_t> xoff;
  std::vector<XinBlock> xb;
  for (const Key4& z : zset) {
    const int m = z[1], c1 = z[2], c2 = z[3];
    if (xoff.count({m, c1, c2})) continue;
    XinBlock b{};
    b.d0 = (int32_t)rcdim[m][c1];
    b.n1 = (int32_t)ncl(c1);
    b.n2 = (int32_t)ncl(c2);
    b.d2 = (int32_t)ccdim[m][c2];
    b.n1p = (int32_t)pad8(b.n1);
    b.n2p = (int32_t)pad8(b.n2);
    b.d2p = (int32_t)pad8(b.d2);
    b.src = H.in_base[m] + rcoff[m][c1] * th.ncols[m] + ccoff[m][c2];
    b.ncols = th.ncols[m];
    b.dst = T->xin_len;
    xoff[{m, c1, c2}] = T->xin_len;
    T->xin_len += align64(pad8(b.d0) * b.n1p * b.n2p * b.d2p);
    T->max_runs = std::max<int64_t>(T->max_runs, (int64_t)b.d0 * b.n1 * b.n2);
    xb.push_back(b);
  }
  if (xb.size() > 65535) return fail(CMPS_ERR_ARG, "canonical tcgen05 form: too many theta blocks");
  T->n_xin = (int)xb.size();
  // ---- MPO class blocks on the host, dense [n_out][n_in], one after another ----
  std::map<Key4, int64_t> wsrc;
  std::vector<double> wre, wim;
  for (auto& wk : wblk) {
    const int ci = wk.first[2], co = wk.first[3];
    const int64_t src = (int64_t)wre.size();
    wsrc[wk.first] = src;
    wre.resize(src + ncl(co) * ncl(ci), 0.0);
    wim.resize(src + ncl(co) * ncl(ci), 0.0);
    for (auto& e : wk.second) {
      wre[(size_t)(src + e.first)] += e.second.first;
      wim[(size_t)(src + e.first)] += e.second.second;
    }
  }
  // ---- intermediates ----
  struct ZInfo {
    int64_t off, rows;  // rows = d0p n1p n2p (the stage-R M)
    int32_t n;          // a2' dim
  };
  std::map<Key4, ZInfo> zinfo;
  int64_t z_len = 0;
  for (const Key4& z : zset) {
    const int b2 = z[0], m = z[1], c1 = z[2], c2 = z[3];
    const int tp = H.R.partner[(size_t)b2 * ns2 + csec[m][c2]];
    ZInfo zi{z_len, pad8(rcdim[m][c1]) * pad8(ncl(c1)) * pad8(ncl(c2)), (int32_t)A2.sdim[tp]};
    zinfo[z] = zi;
    z_len += align64(zi.rows * zi.n);
  }
  struct YInfo {
    int64_t off, rows;  // rows = d2' d0p n1p (the stage-W2 M)
    int32_t n;          // n2' = |c2'|
    std::vector<std::pair<Key4, Key4>> terms;  // (Z key, W key)
  };
  std::map<Key4, YInfo> yinfo;
  int64_t y_len = 0;
  for (const Key4& yk : ycand) {
    const int b1 = yk[0], m = yk[1], c1 = yk[2], c2p = yk[3];
    const int mpp = th.find(r.add(th.mq[m], H.bq[b1]));
    if (mpp < 0 || ccoff[mpp][c2p] < 0) continue;
    YInfo yi{};
    for (auto& wk : wblk) {
      if (wk.first[0] != b1 || wk.first[3] != c2p) continue;
      const Key4 zk{wk.first[1], m, c1, wk.first[2]};
      if (zinfo.count(zk)) yi.terms.push_back({zk, wk.first});
    }
    if (yi.terms.empty()) continue;
    yi.rows = ccdim[mpp][c2p] * pad8(rcdim[m][c1]) * pad8(ncl(c1));
    yi.n = (int32_t)ncl(c2p);
    yi.off = y_len;
    y_len += align64(yi.rows * yi.n);
    yinfo[yk] = std::move(yi);
  }
  struct VInfo {
    int64_t off, rows;  // rows = n2' d2' d0p (the stage-W1 M)
    int32_t n;          // n1' = |c1'|
    int alpha;
    std::vector<std::pair<Key4, Key4>> terms;  // (Y key, W key)
  };
  std::map<VKey, VInfo> vinfo;
  int64_t v_len = 0;
  for (auto& kv : v_alpha) {
    const VKey& v = kv.first;
    VInfo vi{};
    vi.alpha = kv.second;
    for (auto& wk : wblk) {
      if (wk.first[0] != v.b0 || wk.first[3] != v.c1p) continue;
      const int b1 = wk.first[1], c1 = wk.first[2];
      const int m = th.find(r.sub(th.mq[v.mpp], H.bq[b1]));
      if (m < 0) continue;
      const Key4 yk{b1, m, c1, v.c2p};
      if (yinfo.count(yk)) vi.terms.push_back({yk, wk.first});
    }
    if (vi.terms.empty()) continue;
    vi.rows = ncl(v.c2p) * ccdim[v.mpp][v.c2p] * pad8(A0.sdim[vi.alpha]);
    vi.n = (int32_t)ncl(v.c1p);
    vi.off = v_len;
    v_len += align64(vi.rows * vi.n);
    vinfo[v] = std::move(vi);
  }
  T->zv_len = std::max<int64_t>(64, std::max(z_len, v_len));
  T->y_len = std::max<int64_t>(64, y_len);
  T->xin_len = std::max<int64_t>(64, T->xin_len);

  // ---- the stages as raw tasks: output run, A blocks, B source blocks ----
  // A: (buffer 0 Theta_in / 1 Z,V / 2 Y, block offset, K, rows, ld), one map
  // per A block and plan.  B: a block of the R environment (transposed), the
  // L environment or the host-built MPO blocks.
  enum { kSrcR = 0, kSrcL = 1, kSrcW = 2 };
  struct BSrc {
    int src;
    int64_t off;
    int32_t rows, cols, transpose;  // source block rows x cols, row-major
    int32_t n() const { return transpose ? cols : rows; }  // B rows (the task's N)
  };
  struct RawTerm {
    std::array<int64_t, 5> a;  // A block: buffer, offset, K, rows, ld
    int32_t a_y0;
    BSrc b;
  };
  struct RawTask {
    int64_t out_off, col_stride, group;
    int32_t m, n;
    std::vector<RawTerm> terms;
  };
  std::vector<RawTask> rawR, rawW2, rawW1, rawL;
  for (const Key4& z : zset) {
    const int b2 = z[0], m = z[1], c1 = z[2], c2 = z[3];
    const ZInfo& zi = zinfo.at(z);
    const int t = csec[m][c2];
    const int64_t d2 = A2.sdim[t];
    RawTask rt{zi.off, zi.rows, (int64_t)(m * ncls + c1) * ncls + c2, (int32_t)zi.rows, zi.n, {}};
    // R^{b2} stored [a2][a2'] (dim t x dim t'), used as [a2'][a2]
    rt.terms.push_back(RawTerm{{0, xoff.at({m, c1, c2}), d2, zi.rows, pad8(d2)}, 0,
                               BSrc{kSrcR, H.R.off[(size_t)b2 * ns2 + t], (int32_t)d2, zi.n, 1}});
    rawR.push_back(std::move(rt));
  }
  for (auto& kv : yinfo) {
    const Key4& yk = kv.first;
    const YInfo& yi = kv.second;
    RawTask rt{yi.off, yi.rows, (int64_t)yk[1] * ncls + yk[2], (int32_t)yi.rows, yi.n, {}};
    for (auto& tm : yi.terms) {
      const ZInfo& zi = zinfo.at(tm.first);
      const int64_t n2 = ncl(tm.first[3]);
      if (zi.rows / pad8(n2) * zi.n != yi.rows) return fail(CMPS_ERR_STATE, "canonical tcgen05 form: W2 row mismatch");
      rt.terms.push_back(RawTerm{{1, zi.off, n2, yi.rows, pad8(n2)}, 0,
                                 BSrc{kSrcW, wsrc.at(tm.second), yi.n, (int32_t)n2, 0}});
    }
    rawW2.push_back(std::move(rt));
  }
  for (auto& kv : vinfo) {
    const VKey& v = kv.first;
    const VInfo& vi = kv.second;
    RawTask rt{vi.off, vi.rows, (int64_t)v.mpp * ncls + v.c2p, (int32_t)vi.rows, vi.n, {}};
    for (auto& tm : vi.terms) {
      const YInfo& yi = yinfo.at(tm.first);
      const int64_t n1 = ncl(tm.first[2]);
      if (yi.rows / pad8(n1) * yi.n != vi.rows) return fail(CMPS_ERR_STATE, "canonical tcgen05 form: W1 row mismatch");
      rt.terms.push_back(RawTerm{{2, yi.off, n1, vi.rows, pad8(n1)}, 0,
                                 BSrc{kSrcW, wsrc.at(tm.second), vi.n, (int32_t)n1, 0}});
    }
    rawW1.push_back(std::move(rt));
  }
  for (int mpp = 0; mpp < nm; ++mpp)
    for (int c1p = 0; c1p < ncls; ++c1p) {
      if (rcoff[mpp][c1p] < 0) continue;
      const int64_t d0o = rcdim[mpp][c1p];  // a0' dim = N
      for (int c2p = 0; c2p < ncls; ++c2p) {
        if (ccoff[mpp][c2p] < 0) continue;
        const int64_t run = ncl(c2p) * ccdim[mpp][c2p];  // (s2', a2') per s1' = M
        for (int64_t pos = 0; pos < ncl(c1p); ++pos) {
          RawTask rt{H.out_base[mpp] + (rcoff[mpp][c1p] + pos * d0o) * th.ncols[mpp] + ccoff[mpp][c2p],
                     th.ncols[mpp], 0, (int32_t)run, (int32_t)d0o, {}};
          for (int b0 = 0; b0 < H.D; ++b0) {
            auto vit = vinfo.find(VKey{b0, mpp, c1p, c2p});
            if (vit == vinfo.end()) continue;
            const VInfo& vi = vit->second;
            const int64_t d0 = A0.sdim[vi.alpha];
            if (vi.rows != run * pad8(d0) || vi.n != ncl(c1p))
              return fail(CMPS_ERR_STATE, "canonical tcgen05 form: L row mismatch");
            // L^{b0} stored [a0'][a0] (dim a0' x dim a0), used as is
            rt.terms.push_back(RawTerm{{1, vi.off, d0, vi.n * run, pad8(d0)}, (int32_t)(pos * run),
                                       BSrc{kSrcL, H.L.off[(size_t)b0 * ns0 + vi.alpha], (int32_t)d0o, (int32_t)d0, 0}});
          }
          // a task without terms writes zeros; its run inside the output window
          if (rt.out_off < 0 || rt.out_off + (rt.m - 1) + (int64_t)(rt.n - 1) * rt.col_stride >= H.out_len)
            return fail(CMPS_ERR_STATE, "canonical tcgen05 form: output outside theta");
          rawL.push_back(std::move(rt));
        }
      }
    }

  // ---- fusion: tasks with the same A blocks (the same rows, the same K
  // list) become one task of up to four column segments and N <= 128, its
  // B operand the members' B blocks stacked along N.  The MPO stages gain
  // most: on a chain vertex every bond but one reads a single block. ----
  struct FTerm {
    std::array<int64_t, 5> a;
    int32_t a_y0;
    int64_t b_off;  // B block in ops, [N][pad8(K)]
  };
  struct FTask {
    int64_t group, col_stride;
    int32_t m, n, nseg;
    int32_t seg_n0[4];
    int64_t seg_off[4];
    std::vector<FTerm> terms;
  };
  std::vector<SplitBlock> sb[3];
  std::map<std::array<int64_t, 4>, int64_t> bdedup;  // (src, off, transpose, K) of a lone block -> ops offset
  auto b_block = [&](const BSrc& b, int64_t dst, int64_t ld) {
    sb[b.src].push_back(SplitBlock{b.off, dst, b.rows, b.cols, (int32_t)ld, b.transpose});
  };
  auto fuse = [&](std::vector<RawTask>& raw, bool allow, std::vector<FTask>& out) -> int {
    std::map<std::vector<int64_t>, std::vector<size_t>> bysig;
    std::vector<const std::vector<int64_t>*> order;
    for (size_t i = 0; i < raw.size(); ++i) {
      std::vector<int64_t> sig{raw[i].m, raw[i].group};
      for (const RawTerm& t : raw[i].terms) {
        sig.insert(sig.end(), t.a.begin(), t.a.end());
        sig.push_back(t.a_y0);
      }
      if (!allow) sig.push_back((int64_t)i);
      auto it = bysig.find(sig);
      if (it == bysig.end()) {
        it = bysig.emplace(sig, std::vector<size_t>()).first;
        order.push_back(&it->first);
      }
      it->second.push_back(i);
    }
    for (const std::vector<int64_t>* sig : order) {
      const std::vector<size_t>& mem = bysig.at(*sig);
      size_t i = 0;
      while (i < mem.size()) {
        // members of this task: consecutive ones while N <= 128 and <= 4 segments
        std::vector<size_t> part{mem[i++]};
        int32_t ntot = raw[part[0]].n;
        while (i < mem.size() && raw[part[0]].n <= 64 && raw[mem[i]].n <= 64 && part.size() < 4 &&
               ntot + raw[mem[i]].n <= 128) {
          ntot += raw[mem[i]].n;
          part.push_back(mem[i++]);
        }
        const RawTask& r0 = raw[part[0]];
        FTask f{r0.group, r0.col_stride, r0.m, ntot, (int32_t)part.size(), {}, {}, {}};
        int32_t col = 0;
        for (int q = 0; q < 4; ++q) {
          f.seg_n0[q] = q < f.nseg ? col : 0x7fffffff;
          f.seg_off[q] = q < f.nseg ? raw[part[q]].out_off : 0;
          if (q < f.nseg) {
            if (raw[part[q]].col_stride != f.col_stride) return fail(CMPS_ERR_STATE, "canonical tcgen05 form: fusion");
            col += raw[part[q]].n;
          }
        }
        for (size_t q = 0; q < r0.terms.size(); ++q) {
          const int64_t K = r0.terms[q].a[2], ld = pad8(K);
          int64_t off;
          if (part.size() == 1) {
            const BSrc& b = r0.terms[q].b;
            const std::array<int64_t, 4> key{b.src, b.off, b.transpose, K};
            auto it = bdedup.find(key);
            if (it != bdedup.end()) {
              off = it->second;
            } else {
              off = T->ops_len;
              b_block(b, off, ld);
              T->ops_len += align64((int64_t)b.n() * ld);
              bdedup[key] = off;
            }
          } else {
            off = T->ops_len;
            int64_t row = 0;
            for (size_t s : part) {
              const BSrc& b = raw[s].terms[q].b;
              b_block(b, off + row * ld, ld);
              row += b.n();
            }
            T->ops_len += align64(ntot * ld);
          }
          f.terms.push_back(FTerm{r0.terms[q].a, r0.terms[q].a_y0, off});
        }
        out.push_back(std::move(f));
      }
    }
    return CMPS_OK;
  };
  std::vector<FTask> fR, fW2, fW1, fL;
  CMPS_TRY(fuse(rawR, true, fR));
  CMPS_TRY(fuse(rawW2, true, fW2));
  CMPS_TRY(fuse(rawW1, true, fW1));
  CMPS_TRY(fuse(rawL, false, fL));
  T->ops_len = std::max<int64_t>(64, T->ops_len);

  // ---- device buffers: the intermediates inside the FP64 canonical ones
  // when they fit (the FP64 and split matvecs never run at once) ----
  auto fits = [](const Planar& p, int64_t len) { return p.d && 8 * len <= 16 * p.len; };
  if (fits(*fp64_xz, T->zv_len)) {
    T->zv = (uint16_t*)fp64_xz->d;
  } else {
    CMPS_CUDA(dmalloc(&T->zv, (size_t)8 * T->zv_len));
    T->own_zv = true;
  }
  if (fits(*fp64_y, T->y_len)) {
    T->y = (uint16_t*)fp64_y->d;
  } else {
    CMPS_CUDA(dmalloc(&T->y, (size_t)8 * T->y_len));
    T->own_y = true;
  }
  CMPS_CUDA(dmalloc(&T->xin, (size_t)8 * T->xin_len));
  CMPS_CUDA(dmalloc(&T->ops, (size_t)8 * T->ops_len));
  CMPS_CUDA(cudaMemsetAsync(T->xin, 0, (size_t)8 * T->xin_len, st));  // the padding stays zero
  CMPS_CUDA(cudaMemsetAsync(T->ops, 0, (size_t)8 * T->ops_len, st));
  if (!xb.empty()) {
    CMPS_CUDA(dmalloc(&T->d_xin, sizeof(XinBlock) * xb.size()));
    CMPS_TRY(copy_wait(T->d_xin, xb.data(), sizeof(XinBlock) * xb.size(), cudaMemcpyHostToDevice, st));
  }
  CMPS_CUDA(dmalloc(&T->d_err, sizeof(int)));
  CMPS_CUDA(cudaMemsetAsync(T->d_err, 0, sizeof(int), st));
  CMPS_CUDA(cudaMallocHost(&T->h_err, sizeof(int)));
  *T->h_err = 0;
  // ---- split the B operands ----
  {
    Planar wdev;
    if (!wre.empty()) {
      CMPS_TRY(wdev.alloc((int64_t)wre.size()));
      CMPS_TRY(copy_wait(wdev.re(), wre.data(), sizeof(double) * wre.size(), cudaMemcpyHostToDevice, st));
      CMPS_TRY(copy_wait(wdev.im(), wim.data(), sizeof(double) * wim.size(), cudaMemcpyHostToDevice, st));
    }
    for (int pass = 0; pass < 3; ++pass) {
      const std::vector<SplitBlock>& v = sb[pass];
      const Planar& src = pass == kSrcR ? H.R.data : pass == kSrcL ? H.L.data : wdev;
      if (v.empty()) continue;
      for (const SplitBlock& b : v)
        if (b.src_off < 0 || b.src_off + (int64_t)b.rows * b.cols > src.len || b.dst_off < 0 ||
            b.dst_off + (int64_t)((b.transpose ? b.cols : b.rows) - 1) * b.ld_dst + (b.transpose ? b.rows : b.cols) >
                T->ops_len)
          return fail(CMPS_ERR_STATE, "canonical tcgen05 form: operand block outside its buffer");
      SplitBlock* d = nullptr;
      CMPS_CUDA(dmalloc(&d, sizeof(SplitBlock) * v.size()));
      int rc = copy_wait(d, v.data(), sizeof(SplitBlock) * v.size(), cudaMemcpyHostToDevice, st);
      if (rc == CMPS_OK) {
        k_split_blocks<uint16_t><<<(unsigned)v.size(), 256, 0, st>>>(d, src.re(), src.im(), T->ops, T->ops_len);
        if (cudaGetLastError() != cudaSuccess) rc = fail(CMPS_ERR_CUDA, "operand split launch failed");
      }
      if (rc == CMPS_OK && cudaStreamSynchronize(st) != cudaSuccess) rc = fail(CMPS_ERR_CUDA, "operand split failed");
      dfree(d);
      if (rc != CMPS_OK) return rc;
    }
  }
  // ---- plans: tensor maps, tasks, tiles ----
  const uint16_t* abuf[3] = {T->xin, T->zv, T->y};
  const int64_t alen[3] = {T->xin_len, T->zv_len, T->y_len};
  auto build_plan = [&](tc::TcPlan& p, std::vector<FTask>& ft, bool grouped, const uint16_t* out,
                        int64_t out_len) -> int {
    std::map<std::array<int64_t, 5>, int32_t> amaps;
    std::map<std::array<int64_t, 3>, int32_t> bmaps;  // (ops offset, K, rows)
    std::vector<int32_t> brows;
    std::map<int64_t, std::vector<int32_t>> groups;
    for (const FTask& f : ft) {
      tc::TcTask task{};
      task.out_off = f.seg_off[0];
      task.row_stride = 1;
      task.col_stride = f.col_stride;
      task.m = f.m;
      task.n = f.n;
      task.nseg = f.nseg;
      for (int q = 0; q < 4; ++q) {
        task.seg_n0[q] = f.seg_n0[q];
        task.seg_off[q] = f.seg_off[q];
      }
      // every segment's run inside the output buffer
      for (int q = 0; q < f.nseg; ++q) {
        const int32_t nq = (q + 1 < f.nseg ? f.seg_n0[q + 1] : f.n) - f.seg_n0[q];
        if (f.seg_off[q] < 0 || f.seg_off[q] + (f.m - 1) + (int64_t)(nq - 1) * f.col_stride >= out_len)
          return fail(CMPS_ERR_STATE, "canonical tcgen05 form: output outside its buffer");
      }
      task.t0 = (int32_t)p.terms.size();
      for (const FTerm& t : f.terms) {
        int32_t a, b;
        auto ia = amaps.find(t.a);
        if (ia != amaps.end()) {
          a = ia->second;
        } else {
          const int buf = (int)t.a[0];
          CUtensorMap cm;
          CMPS_TRY(tc::encode_map(true, abuf[buf] + t.a[1], t.a[2], t.a[3], t.a[4], alen[buf], alen[buf] - t.a[1], 128,
                                  &cm));
          a = (int32_t)p.amaps.size();
          p.amaps.push_back(cm);
          amaps[t.a] = a;
        }
        const std::array<int64_t, 3> bk{t.b_off, t.a[2], f.n};
        auto ib = bmaps.find(bk);
        if (ib != bmaps.end()) {
          b = ib->second;
        } else {
          CUtensorMap cm;
          CMPS_TRY(tc::encode_map(true, T->ops + t.b_off, t.a[2], f.n, pad8(t.a[2]), T->ops_len, T->ops_len - t.b_off,
                                  tc::b_box_rows(f.n), &cm));
          b = (int32_t)p.bmaps.size();
          p.bmaps.push_back(cm);
          brows.push_back(f.n);
          bmaps[bk] = b;
        }
        tc::TcTerm tm{a, b, 0, (int32_t)t.a[2]};
        tm.a_y0 = t.a_y0;
        p.terms.push_back(tm);
        T->flops += 8.0 * f.m * (double)f.n * t.a[2];
      }
      task.t1 = (int32_t)p.terms.size();
      if (grouped)
        groups[f.group].push_back((int32_t)p.tasks.size());
      else
        tc::add_tiles(p, (int32_t)p.tasks.size(), task.m, task.n);
      p.tasks.push_back(task);
    }
    // Tiles of a group of tasks that read the same A rows go row tile by row
    // tile across the group, so the tiles that run at the same time (dealt
    // round-robin to the SMs) share their A tiles in L2.
    for (auto& g : groups) {
      int32_t mmax = 0;
      for (int32_t t : g.second) mmax = std::max(mmax, p.tasks[t].m);
      for (int32_t m0 = 0; m0 < mmax; m0 += 128)
        for (int32_t t : g.second) {
          const tc::TcTask& k = p.tasks[t];
          if (m0 >= k.m) continue;
          for (int32_t n0 = 0; n0 < k.n; n0 += 128)
            p.tiles.push_back(tc::TcTile{t, m0, n0, tc::b_box_rows(k.n), 0, ((std::min(128, k.n - n0)) + 15) & ~15});
        }
    }
    if (out) tc::mark_vector_stores(p, out, out_len);  // mode 3: BF16 output in 16-byte stores
    return tc::finish_plan(p, true, true, brows, !grouped, true);
  };
  CMPS_TRY(build_plan(T->pR, fR, true, T->zv, T->zv_len));
  CMPS_TRY(build_plan(T->pW2, fW2, true, T->y, T->y_len));
  CMPS_TRY(build_plan(T->pW1, fW1, true, T->zv, T->zv_len));
  CMPS_TRY(build_plan(T->pL, fL, false, nullptr, H.out_len));
  for (tc::TcPlan* p : {&T->pR, &T->pW2, &T->pW1, &T->pL}) CMPS_TRY(p->upload(st));
  CMPS_CUDA(cudaStreamSynchronize(st));
  return CMPS_OK;
}

// which: 1 = theta in, stages R and W2; 2 = stages W1 and L; 0 = all.
int apply_canonical_tc(Heff& H, int which, const Planar& in, Planar& out, cudaStream_t st) {
  CanonTc* T = H.ctc;
  if (!T) return fail(CMPS_ERR_STATE, "canonical tcgen05 form not prepared");
  if (which != 2) {
    if (T->n_xin > 0 && T->max_runs > 0) {
      const int64_t gx = std::min<int64_t>((T->max_runs + 7) / 8, 2048);
      k_gather_theta<<<dim3((unsigned)gx, (unsigned)T->n_xin), 256, 0, st>>>(T->d_xin, in.re(), in.im(), T->xin,
                                                                             T->xin_len);
      CMPS_CUDA(cudaGetLastError());
    }
    CMPS_TRY(tc::launch(3, T->pR, (float*)T->zv, T->zv_len, nullptr, 0, nullptr, 0, T->d_err, st));
    CMPS_TRY(tc::launch(3, T->pW2, (float*)T->y, T->y_len, nullptr, 0, nullptr, 0, T->d_err, st));
  }
  if (which != 1) {
    CMPS_TRY(tc::launch(3, T->pW1, (float*)T->zv, T->zv_len, nullptr, 0, nullptr, 0, T->d_err, st));
    CMPS_TRY(tc::launch(4, T->pL, nullptr, 0, out.re(), out.len, nullptr, 0, T->d_err, st));
  }
  return CMPS_OK;
}

double canonical_tc_flops(const Heff& H) { return H.ctc ? H.ctc->flops : 0.0; }

}  // namespace cmps
