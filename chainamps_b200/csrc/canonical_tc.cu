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
  // ---- B operand blocks: R^T (b2, t), W (bl, br, ci, co), L (b0, s) ----
  std::map<std::array<int, 2>, int64_t> roff, loff;
  std::map<Key4, int64_t> woff;
  std::vector<SplitBlock> rsb, lsb, wsb;
  std::vector<double> wre, wim;  // dense W blocks, contiguous [n_out][n_in]
  for (const Key4& z : zset) {
    const int b2 = z[0], t = csec[z[1]][z[3]];
    if (roff.count({b2, t})) continue;
    const int tp = H.R.partner[(size_t)b2 * ns2 + t];
    roff[{b2, t}] = T->ops_len;
    // stored [a2][a2'] (dim t x dim t'); wanted [a2'][a2], ld pad8(dim t)
    rsb.push_back(SplitBlock{H.R.off[(size_t)b2 * ns2 + t], T->ops_len, (int32_t)A2.sdim[t], (int32_t)A2.sdim[tp],
                             (int32_t)pad8(A2.sdim[t]), 1});
    T->ops_len += align64(A2.sdim[tp] * pad8(A2.sdim[t]));
  }
  for (auto& wk : wblk) {
    const int ci = wk.first[2], co = wk.first[3];
    woff[wk.first] = T->ops_len;
    const int64_t src = (int64_t)wre.size();
    wre.resize(src + ncl(co) * ncl(ci), 0.0);
    wim.resize(src + ncl(co) * ncl(ci), 0.0);
    for (auto& e : wk.second) {
      wre[(size_t)(src + e.first)] += e.second.first;
      wim[(size_t)(src + e.first)] += e.second.second;
    }
    wsb.push_back(SplitBlock{src, T->ops_len, (int32_t)ncl(co), (int32_t)ncl(ci), (int32_t)pad8(ncl(ci)), 0});
    T->ops_len += align64(ncl(co) * pad8(ncl(ci)));
  }
  for (auto& kv : v_alpha) {
    const int b0 = kv.first.b0, s = kv.second;
    if (loff.count({b0, s})) continue;
    const int sp = H.L.partner[(size_t)b0 * ns0 + s];
    loff[{b0, s}] = T->ops_len;
    // stored [a0'][a0] (dim s' x dim s), kept as is with ld pad8(dim s)
    lsb.push_back(SplitBlock{H.L.off[(size_t)b0 * ns0 + s], T->ops_len, (int32_t)A0.sdim[sp], (int32_t)A0.sdim[s],
                             (int32_t)pad8(A0.sdim[s]), 0});
    T->ops_len += align64(A0.sdim[sp] * pad8(A0.sdim[s]));
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
      const std::vector<SplitBlock>& v = pass == 0 ? rsb : pass == 1 ? lsb : wsb;
      const Planar& src = pass == 0 ? H.R.data : pass == 1 ? H.L.data : wdev;
      if (v.empty()) continue;
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
  // ---- plans ----
  std::map<std::pair<int64_t, int>, int32_t> bmap_of;  // (ops offset, K) -> B map index, per plan
  std::vector<int32_t> brows;
  auto bmap = [&](tc::TcPlan& p, int64_t off, int64_t K, int64_t rows, int64_t ld, int32_t* out) -> int {
    auto it = bmap_of.find({off, (int)K});
    if (it != bmap_of.end()) {
      *out = it->second;
      return CMPS_OK;
    }
    CUtensorMap cm;
    CMPS_TRY(tc::encode_map(true, T->ops + off, K, rows, ld, T->ops_len, T->ops_len - off,
                            tc::b_box_rows((int32_t)rows), &cm));
    *out = (int32_t)p.bmaps.size();
    p.bmaps.push_back(cm);
    brows.push_back((int32_t)rows);
    bmap_of[{off, (int)K}] = *out;
    return CMPS_OK;
  };
  auto amap = [&](tc::TcPlan& p, const uint16_t* buf, int64_t plane, int64_t off, int64_t K, int64_t rows, int64_t ld,
                  int32_t* out) -> int {
    CUtensorMap cm;
    CMPS_TRY(tc::encode_map(true, buf + off, K, rows, ld, plane, plane - off, 128, &cm));
    *out = (int32_t)p.amaps.size();
    p.amaps.push_back(cm);
    return CMPS_OK;
  };
  auto one_segment = [](tc::TcTask& t, int64_t off) {
    t.out_off = off;
    t.nseg = 1;
    t.seg_n0[0] = 0;
    t.seg_off[0] = off;
    for (int q = 1; q < 4; ++q) {
      t.seg_n0[q] = 0x7fffffff;
      t.seg_off[q] = 0;
    }
  };
  // Tiles of a group of tasks that read the same A rows: row tile by row
  // tile across the group, so the tiles that run at the same time (dealt
  // round-robin to the SMs) share their A tiles in L2.
  auto group_tiles = [](tc::TcPlan& p, const std::vector<int32_t>& group) {
    int32_t mmax = 0;
    for (int32_t t : group) mmax = std::max(mmax, p.tasks[t].m);
    for (int32_t m0 = 0; m0 < mmax; m0 += 128)
      for (int32_t t : group) {
        const tc::TcTask& k = p.tasks[t];
        if (m0 >= k.m) continue;
        for (int32_t n0 = 0; n0 < k.n; n0 += 128)
          p.tiles.push_back(tc::TcTile{t, m0, n0, tc::b_box_rows(k.n), 0, ((std::min(128, k.n - n0)) + 15) & ~15});
      }
  };
  auto term_flops = [](const tc::TcTask& t, int64_t k) { return 8.0 * t.m * (double)t.n * k; };

  // stage R: Z^{b2}_{m,c1,c2}[a2'][rows] = Theta_in[rows][a2] . R^T[a2'][a2]
  {
    tc::TcPlan& p = T->pR;
    bmap_of.clear();
    brows.clear();
    std::map<std::array<int, 3>, int32_t> xa;
    std::map<std::array<int, 3>, std::vector<int32_t>> groups;
    for (const Key4& z : zset) {
      const int b2 = z[0], m = z[1], c1 = z[2], c2 = z[3];
      const ZInfo& zi = zinfo.at(z);
      const int t = csec[m][c2];
      const int64_t d2 = A2.sdim[t];
      auto it = xa.find({m, c1, c2});
      int32_t a;
      if (it == xa.end()) {
        CMPS_TRY(amap(p, T->xin, T->xin_len, xoff.at({m, c1, c2}), d2, zi.rows, pad8(d2), &a));
        xa[{m, c1, c2}] = a;
      } else {
        a = it->second;
      }
      int32_t b;
      CMPS_TRY(bmap(p, roff.at({b2, t}), d2, zi.n, pad8(d2), &b));
      tc::TcTask task{};
      one_segment(task, zi.off);
      task.row_stride = 1;
      task.col_stride = zi.rows;
      task.m = (int32_t)zi.rows;
      task.n = zi.n;
      task.t0 = (int32_t)p.terms.size();
      p.terms.push_back(tc::TcTerm{a, b, 0, (int32_t)d2});
      task.t1 = (int32_t)p.terms.size();
      T->flops += term_flops(task, d2);
      groups[{m, c1, c2}].push_back((int32_t)p.tasks.size());
      p.tasks.push_back(task);
    }
    for (auto& g : groups) group_tiles(p, g.second);
    CMPS_TRY(tc::finish_plan(p, true, true, brows, false));
  }
  // stage W2: Y^{b1}_{m,c1,c2'}[s2'][rows] = sum Z^{b2}_{m,c1,c2}[rows][s2] . W[s2'][s2]
  {
    tc::TcPlan& p = T->pW2;
    bmap_of.clear();
    brows.clear();
    std::map<Key4, int32_t> za;
    std::map<std::pair<int, int>, std::vector<int32_t>> groups;
    for (auto& kv : yinfo) {
      const Key4& yk = kv.first;
      const YInfo& yi = kv.second;
      tc::TcTask task{};
      one_segment(task, yi.off);
      task.row_stride = 1;
      task.col_stride = yi.rows;
      task.m = (int32_t)yi.rows;
      task.n = yi.n;
      task.t0 = (int32_t)p.terms.size();
      for (auto& tm : yi.terms) {
        const Key4& zk = tm.first;
        const ZInfo& zi = zinfo.at(zk);
        const int64_t n2 = ncl(zk[3]);
        if (zi.rows / pad8(n2) * zi.n != yi.rows) return fail(CMPS_ERR_STATE, "canonical tcgen05 form: W2 row mismatch");
        int32_t a;
        auto it = za.find(zk);
        if (it == za.end()) {
          CMPS_TRY(amap(p, T->zv, T->zv_len, zi.off, n2, yi.rows, pad8(n2), &a));
          za[zk] = a;
        } else {
          a = it->second;
        }
        int32_t b;
        CMPS_TRY(bmap(p, woff.at(tm.second), n2, yi.n, pad8(n2), &b));
        p.terms.push_back(tc::TcTerm{a, b, 0, (int32_t)n2});
        T->flops += term_flops(task, n2);
      }
      task.t1 = (int32_t)p.terms.size();
      groups[{yk[1], yk[2]}].push_back((int32_t)p.tasks.size());
      p.tasks.push_back(task);
    }
    for (auto& g : groups) group_tiles(p, g.second);
    CMPS_TRY(tc::finish_plan(p, true, true, brows, false));
  }
  // stage W1: V^{b0}_{m'',c1',c2'}[s1'][rows] = sum Y^{b1}_{m,c1,c2'}[rows][s1] . W[s1'][s1]
  {
    tc::TcPlan& p = T->pW1;
    bmap_of.clear();
    brows.clear();
    std::map<Key4, int32_t> ya;
    std::map<std::pair<int, int>, std::vector<int32_t>> groups;
    for (auto& kv : vinfo) {
      const VKey& v = kv.first;
      const VInfo& vi = kv.second;
      tc::TcTask task{};
      one_segment(task, vi.off);
      task.row_stride = 1;
      task.col_stride = vi.rows;
      task.m = (int32_t)vi.rows;
      task.n = vi.n;
      task.t0 = (int32_t)p.terms.size();
      for (auto& tm : vi.terms) {
        const Key4& yk = tm.first;
        const YInfo& yi = yinfo.at(yk);
        const int64_t n1 = ncl(yk[2]);
        if (yi.rows / pad8(n1) * yi.n != vi.rows) return fail(CMPS_ERR_STATE, "canonical tcgen05 form: W1 row mismatch");
        int32_t a;
        auto it = ya.find(yk);
        if (it == ya.end()) {
          CMPS_TRY(amap(p, T->y, T->y_len, yi.off, n1, vi.rows, pad8(n1), &a));
          ya[yk] = a;
        } else {
          a = it->second;
        }
        int32_t b;
        CMPS_TRY(bmap(p, woff.at(tm.second), n1, vi.n, pad8(n1), &b));
        p.terms.push_back(tc::TcTerm{a, b, 0, (int32_t)n1});
        T->flops += term_flops(task, n1);
      }
      task.t1 = (int32_t)p.terms.size();
      groups[{v.mpp, v.c2p}].push_back((int32_t)p.tasks.size());
      p.tasks.push_back(task);
    }
    for (auto& g : groups) group_tiles(p, g.second);
    CMPS_TRY(tc::finish_plan(p, true, true, brows, false));
  }
  // stage L: Theta'_{m''}[(s1', a0')][(s2', a2')] = sum_b0 V^{b0}[s1'][(s2', a2')][a0] . L^{b0}[a0'][a0]
  {
    tc::TcPlan& p = T->pL;
    bmap_of.clear();
    brows.clear();
    std::map<VKey, int32_t> va;
    for (int mpp = 0; mpp < nm; ++mpp)
      for (int c1p = 0; c1p < ncls; ++c1p) {
        if (rcoff[mpp][c1p] < 0) continue;
        const int64_t d0o = rcdim[mpp][c1p];  // a0' dim = N
        for (int c2p = 0; c2p < ncls; ++c2p) {
          if (ccoff[mpp][c2p] < 0) continue;
          const int64_t run = ncl(c2p) * ccdim[mpp][c2p];  // (s2', a2') per s1' = M
          for (int64_t pos = 0; pos < ncl(c1p); ++pos) {
            tc::TcTask task{};
            one_segment(task, H.out_base[mpp] + (rcoff[mpp][c1p] + pos * d0o) * th.ncols[mpp] + ccoff[mpp][c2p]);
            task.row_stride = 1;
            task.col_stride = th.ncols[mpp];
            task.m = (int32_t)run;
            task.n = (int32_t)d0o;
            task.t0 = (int32_t)p.terms.size();
            for (int b0 = 0; b0 < H.D; ++b0) {
              const VKey vk{b0, mpp, c1p, c2p};
              auto vit = vinfo.find(vk);
              if (vit == vinfo.end()) continue;
              const VInfo& vi = vit->second;
              const int64_t d0 = A0.sdim[vi.alpha];
              if (vi.rows != run * pad8(d0) || vi.n != ncl(c1p))
                return fail(CMPS_ERR_STATE, "canonical tcgen05 form: L row mismatch");
              int32_t a;
              auto it = va.find(vk);
              if (it == va.end()) {
                CMPS_TRY(amap(p, T->zv, T->zv_len, vi.off, d0, vi.n * run, pad8(d0), &a));
                va[vk] = a;
              } else {
                a = it->second;
              }
              int32_t b;
              CMPS_TRY(bmap(p, loff.at({b0, vi.alpha}), d0, d0o, pad8(d0), &b));
              tc::TcTerm tm{a, b, 0, (int32_t)d0};
              tm.a_y0 = (int32_t)(pos * run);
              p.terms.push_back(tm);
              T->flops += term_flops(task, d0);
            }
            task.t1 = (int32_t)p.terms.size();  // a task without terms writes zeros
            // the output run inside the output window
            if (task.out_off < 0 || task.out_off + (task.m - 1) + (int64_t)(task.n - 1) * task.col_stride >= H.out_len)
              return fail(CMPS_ERR_STATE, "canonical tcgen05 form: output outside theta");
            tc::add_tiles(p, (int32_t)p.tasks.size(), task.m, task.n);
            p.tasks.push_back(task);
          }
        }
      }
    CMPS_TRY(tc::finish_plan(p, true, true, brows, true));
  }
  // every intermediate output range inside its buffer
  for (const tc::TcPlan* p : {&T->pR, &T->pW2, &T->pW1}) {
    const int64_t len = p == &T->pW2 ? T->y_len : T->zv_len;
    for (const tc::TcTask& t : p->tasks)
      if (t.out_off + (int64_t)t.m * t.n > len) return fail(CMPS_ERR_STATE, "canonical tcgen05 form: output outside buffer");
  }
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
