// The H_eff matvec in the canonical contraction order, one index at a time:
//
//   X^{b0}_m   = L^{b0} . Theta_m                           (stage L:  contract a0)
//   Y^{b1}_m   = sum_{b0, s1} W[s1', b0, s1, b1] X^{b0}_m     (stage W1: contract sigma1)
//   Z^{b2}_m'' = sum_{b1, s2} W[s2', b1, s2, b2] Y^{b1}_m     (stage W2: contract sigma2)
//   Theta'_m'' = sum_{b2} Z^{b2}_m'' . R^{b2}                  (stage R:  contract a2)
//
// The same linear map as the reference's LeftPart . V . RightPart
// (TwoVertexMPOMPSMultiply, DMRG_routines.cpp:898-945, with LeftPart /
// RightPart from DMRG_routines.cpp:779-806), which folds W into the
// environments.  Folding costs (states per charge class)^2 x the work of one
// environment product per MPO slot; for a vertex with a large local basis
// whose operators are dense inside charge classes (a chain cut to 64 states:
// sigma^x_i fills half of every parity pair) the folded form executes ~28x
// the canonical flops, while for a few-state vertex with sparse operators (a
// spin ladder rung) it is slightly cheaper.  Heff picks the order with the
// fewer executed flops.
//
// Layouts (complex, two planes):
//  * Theta_m: the sector block [(s1, a0)][(s2, a2)], rows and columns grouped
//    by charge class of sigma (Heff::finish), so the rows of one class form
//    n_c equally strided runs of dim(a0-sector) rows, and likewise columns;
//  * X^{b0}_m: rows (s1, a0') class by class (classes whose L block exists),
//    each class n_c x dim(a0') rows; columns those of Theta_m;
//  * Y^{b1}_m: rows of Theta_{m + q(b1)}, columns those of Theta_m;
//  * Z^{b2}_m'': rows of Theta_m'', columns (s2', a2) of charge
//    q(a2) - q(s2') = q(m'') - q(b2) in the class-by-class layout of a theta
//    block (such columns exist even where no theta block of that charge does);
//  * the MPO as one dense block W[., bl, ., br] per (bl, br) and pair of
//    classes: [n_out x n_in].
// Every stage is one grouped FP64 GEMM launch (zgemm_grouped_fp64).  Stage L
// runs one task per (b0, m, class) over all of the class's states with the
// two-level N index; W1 is a plain GEMM over the class's rows; W2 contracts
// sigma2, a column sub-index, with the two-level N index running over
// (row, a2); stage R runs one task per output state sigma2'.  X and Z share
// one buffer (X is dead once W1 has run).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <map>
#include <set>

#include "heff.h"

namespace cmps {

struct Canon {
  Planar ops;    // MPO class blocks
  Planar xz, y;  // intermediates (X then Z; Y)
  GemmPlan sL, sW1, sW2, sR;
  double flops = 0.0;
  // The low-precision form (FP32 planes, the same plans): FP32 copies of the
  // MPO blocks and the environments, theta in and out, and the intermediates
  // as views into the FP64 ones (the two forms never run at once).
  bool have32 = false;
  Planar32 ops32, L32, R32, x32, o32, xz32, y32;
  ~Canon() {
    ops.release();
    xz.release();
    y.release();
    sL.release();
    sW1.release();
    sW2.release();
    sR.release();
    ops32.release();
    L32.release();
    R32.release();
    x32.release();
    o32.release();
  }
};

void release_canonical(Heff* h) {
  release_canonical_tc(h);  // it may borrow the intermediates below
  if (!h || !h->canon) return;
  delete h->canon;
  h->canon = nullptr;
}

namespace {

using Key4 = std::array<int, 4>;

struct Plan {
  // operator blocks: (bl, br, class in, class out) -> offset, [n_out x n_in]
  std::map<Key4, int64_t> opoff;
  int64_t ops_len = 0;
  std::vector<double> ops_re, ops_im;
  // intermediates: (b, m) -> base offset
  std::map<std::pair<int, int>, int64_t> xbase, ybase, zbase;
  std::map<Key4, int64_t> xrow;  // (b0, m, class) -> first row inside X^{b0}_m
  int64_t x_len = 0, y_len = 0, z_len = 0;
  GemmPlan sL, sW1, sW2, sR;
  double flops = 0.0;
  // theta sectors stage L reads; missing: one of them is outside the input window
  std::vector<uint8_t> need;
  bool missing = false;
};

double term_flops(const GemmTask& t, const GemmTerm& tm) { return 8.0 * t.m * (double)t.n * tm.k; }

}  // namespace

// Builds the four stage plans (host side) for the owned output sectors.
static int plan_canonical(const Heff& H, Plan& P) {
  const Rules& r = H.rules;
  const ThetaSpace& th = H.th;
  const Bond& A0 = H.L.a;
  const Bond& A2 = H.R.a;
  const int nm = (int)th.mq.size();
  const int ncls = (int)H.cls_mem.size();
  const int ns0 = A0.nsec(), ns2 = A2.nsec();
  // per (m, class): first row / column of the class and rows / columns per state
  std::vector<std::vector<int64_t>> rcoff(nm, std::vector<int64_t>(ncls, -1)), rcdim = rcoff;
  std::vector<std::vector<int64_t>> ccoff = rcoff, ccdim = rcoff;
  for (int m = 0; m < nm; ++m)
    for (int c = 0; c < ncls; ++c) {
      const std::vector<int>& mem = H.cls_mem[c];
      const QKey qc = H.sigq[mem[0]];
      if (th.rowoff[m][mem[0]] >= 0) {
        rcoff[m][c] = th.rowoff[m][mem[0]];
        rcdim[m][c] = A0.sdim[A0.find(r.sub(th.mq[m], qc))];
        for (size_t i = 0; i < mem.size(); ++i)
          if (th.rowoff[m][mem[i]] != rcoff[m][c] + (int64_t)i * rcdim[m][c])
            return fail(CMPS_ERR_STATE, "canonical order: class rows not equally strided");
      }
      if (th.coloff[m][mem[0]] >= 0) {
        ccoff[m][c] = th.coloff[m][mem[0]];
        ccdim[m][c] = A2.sdim[A2.find(r.add(th.mq[m], qc))];
        for (size_t i = 0; i < mem.size(); ++i)
          if (th.coloff[m][mem[i]] != ccoff[m][c] + (int64_t)i * ccdim[m][c])
            return fail(CMPS_ERR_STATE, "canonical order: class columns not equally strided");
      }
    }
  // Column layout of any middle charge mu, class by class: Z^{b2}_m'' carries
  // the columns (s2', a2) with q(a2) - q(s2') = q(m'') - q(b2), a charge whose
  // row side need not exist, so it need not be a theta block.  For a theta
  // block the layout is the block's own (same class order, same sectors).
  struct ColLayout {
    int64_t n = 0;
    std::vector<int64_t> off, dim;  // per class, -1 if absent
  };
  std::map<QKey, ColLayout> colcache;
  auto collayout = [&](const QKey& mu) -> const ColLayout& {
    auto it = colcache.find(mu);
    if (it != colcache.end()) return it->second;
    ColLayout cl;
    cl.off.assign(ncls, -1);
    cl.dim.assign(ncls, -1);
    for (int c = 0; c < ncls; ++c) {
      const int t = A2.find(r.add(mu, H.sigq[H.cls_mem[c][0]]));
      if (t < 0) continue;
      cl.off[c] = cl.n;
      cl.dim[c] = A2.sdim[t];
      cl.n += (int64_t)H.cls_mem[c].size() * A2.sdim[t];
    }
    return colcache.emplace(mu, std::move(cl)).first->second;
  };
  for (int m = 0; m < nm; ++m) {
    const ColLayout& cl = collayout(th.mq[m]);
    if (cl.n != th.ncols[m] || cl.off != ccoff[m]) return fail(CMPS_ERR_STATE, "canonical order: column layout mismatch");
  }
  // ---- operator blocks ----
  for (const WEntry& w : H.W) {
    Key4 k{w.bl, w.br, H.cls_of[w.s], H.cls_of[w.sp]};
    if (P.opoff.count(k)) continue;
    P.opoff[k] = P.ops_len;
    P.ops_len += (int64_t)H.cls_mem[k[3]].size() * (int64_t)H.cls_mem[k[2]].size();
  }
  P.ops_re.assign((size_t)std::max<int64_t>(P.ops_len, 1), 0.0);
  P.ops_im = P.ops_re;
  for (const WEntry& w : H.W) {
    const int ci = H.cls_of[w.s], co = H.cls_of[w.sp];
    const int64_t o = P.opoff.at({w.bl, w.br, ci, co}) + (int64_t)H.cls_pos[w.sp] * (int64_t)H.cls_mem[ci].size() +
                      H.cls_pos[w.s];
    P.ops_re[(size_t)o] += w.wr;
    P.ops_im[(size_t)o] += w.wi;
  }
  // op pairs by (bl, br): list of (ci, co)
  std::map<std::pair<int, int>, std::vector<std::pair<int, int>>> pairs;
  for (auto& kv : P.opoff) pairs[{kv.first[0], kv.first[1]}].push_back({kv.first[2], kv.first[3]});

  // ---- what is needed, from the owned outputs backwards ----
  // Z^{b2}_m'': m'' owned, columns of charge q(m'') - q(b2) exist, R has blocks for b2
  std::set<int> br_used;
  for (const WEntry& w : H.W) br_used.insert(w.br);
  std::set<std::pair<int, int>> zneed, yneed, xneed;
  for (int mpp = 0; mpp < nm; ++mpp) {
    if (!H.owned[mpp]) continue;
    for (int b2 : br_used) {
      if (collayout(r.sub(th.mq[mpp], H.bq[b2])).n == 0) continue;
      bool any = false;
      for (int t = 0; t < ns2 && !any; ++t) any = H.R.off[(size_t)b2 * ns2 + t] >= 0;
      if (any) zneed.insert({b2, mpp});
    }
  }
  for (auto& z : zneed)
    for (auto& pr : pairs) {
      if (pr.first.second != z.first) continue;
      const int b1 = pr.first.first;
      const int m = th.find(r.sub(th.mq[z.second], H.bq[b1]));
      if (m >= 0) yneed.insert({b1, m});
    }
  for (auto& yv : yneed)
    for (auto& pr : pairs) {
      if (pr.first.second != yv.first) continue;
      xneed.insert({pr.first.first, yv.second});
    }
  // ---- X layout ----
  for (auto& xv : xneed) {
    const int b0 = xv.first, m = xv.second;
    int64_t rows = 0;
    for (int c = 0; c < ncls; ++c) {
      if (rcoff[m][c] < 0) continue;
      const int s = A0.find(r.sub(th.mq[m], H.sigq[H.cls_mem[c][0]]));
      if (H.L.off[(size_t)b0 * ns0 + s] < 0) continue;
      const int sp = H.L.partner[(size_t)b0 * ns0 + s];
      P.xrow[{b0, m, c, 0}] = rows;
      rows += (int64_t)H.cls_mem[c].size() * A0.sdim[sp];
    }
    if (!rows) continue;
    P.xbase[xv] = P.x_len;
    P.x_len += rows * th.ncols[m];
  }
  for (auto& yv : yneed) {
    const int mp = th.find(r.add(th.mq[yv.second], H.bq[yv.first]));
    if (mp < 0) continue;
    P.ybase[yv] = P.y_len;
    P.y_len += th.nrows[mp] * th.ncols[yv.second];
  }
  for (auto& z : zneed) {
    P.zbase[z] = P.z_len;
    P.z_len += th.nrows[z.second] * collayout(r.sub(th.mq[z.second], H.bq[z.first])).n;
  }
  // ---- stage L: X^{b0}_m[class c] = L^{b0} . Theta_m[class c rows] ----
  P.sL.nsplit = true;
  for (auto& xb : P.xbase) {
    const int b0 = xb.first.first, m = xb.first.second;
    const int64_t nc = th.ncols[m];
    for (int c = 0; c < ncls; ++c) {
      auto it = P.xrow.find({b0, m, c, 0});
      if (it == P.xrow.end()) continue;
      const int s = A0.find(r.sub(th.mq[m], H.sigq[H.cls_mem[c][0]]));
      const int sp = H.L.partner[(size_t)b0 * ns0 + s];
      const int64_t n_c = (int64_t)H.cls_mem[c].size();
      GemmTask t{};
      t.c_off = xb.second + it->second * nc;
      t.m = (int32_t)A0.sdim[sp];
      t.n = (int32_t)(n_c * nc);
      t.ldc = (int32_t)nc;
      t.n_in = (int32_t)nc;
      t.ldc_out = (int32_t)(A0.sdim[sp] * nc);
      t.t0 = (int32_t)P.sL.terms.size();
      GemmTerm tm{};
      tm.a_off = H.L.off[(size_t)b0 * ns0 + s];
      tm.lda = (int32_t)A0.sdim[s];
      tm.k = (int32_t)A0.sdim[s];
      if ((int)P.need.size() != nm) P.need.assign(nm, 0);
      P.need[m] = 1;
      if (H.in_base[m] < 0) P.missing = true;
      tm.b_off = std::max<int64_t>(0, H.in_base[m]) + rcoff[m][c] * nc;
      tm.ldb = (int32_t)nc;
      tm.ldb_out = (int32_t)(rcdim[m][c] * nc);
      P.sL.terms.push_back(tm);
      t.t1 = (int32_t)P.sL.terms.size();
      P.flops += term_flops(t, tm);
      P.sL.tasks.push_back(t);
    }
  }
  // ---- stage W1: Y^{b1}_m[class c' rows] = sum W-block . X^{b0}_m[class c rows] ----
  for (auto& yb : P.ybase) {
    const int b1 = yb.first.first, m = yb.first.second;
    const int mp = th.find(r.add(th.mq[m], H.bq[b1]));
    const int64_t nc = th.ncols[m];
    for (int co = 0; co < ncls; ++co) {
      if (rcoff[mp][co] < 0) continue;
      const int64_t n_o = (int64_t)H.cls_mem[co].size();
      const int64_t span = rcdim[mp][co] * nc;  // one state's rows, all columns
      GemmTask t{};
      t.c_off = yb.second + rcoff[mp][co] * nc;
      t.m = (int32_t)n_o;
      t.n = (int32_t)span;
      t.ldc = (int32_t)span;
      t.t0 = (int32_t)P.sW1.terms.size();
      for (auto& kv : P.opoff) {
        const int b0 = kv.first[0];
        if (kv.first[1] != b1 || kv.first[3] != co) continue;
        const int ci = kv.first[2];
        auto xb = P.xbase.find({b0, m});
        if (xb == P.xbase.end()) continue;
        auto xr = P.xrow.find({b0, m, ci, 0});
        if (xr == P.xrow.end()) continue;
        // X rows of class ci carry a0' of sector m - q(ci) + q(b0) = m' - q(co)
        const int s = A0.find(r.sub(th.mq[m], H.sigq[H.cls_mem[ci][0]]));
        if (H.L.partner[(size_t)b0 * ns0 + s] != A0.find(r.sub(th.mq[mp], H.sigq[H.cls_mem[co][0]])))
          return fail(CMPS_ERR_STATE, "canonical order: W1 sector mismatch");
        GemmTerm tm{};
        tm.a_off = kv.second;
        tm.lda = (int32_t)H.cls_mem[ci].size();
        tm.k = (int32_t)H.cls_mem[ci].size();
        tm.b_off = xb->second + xr->second * nc;
        tm.ldb = (int32_t)span;
        P.sW1.terms.push_back(tm);
        P.flops += term_flops(t, tm);
      }
      t.t1 = (int32_t)P.sW1.terms.size();
      P.sW1.tasks.push_back(t);  // a task without terms writes zeros
    }
  }
  // ---- stage W2: Z^{b2}_m''[., class c2' columns] = sum W-block . Y^{b1}_m[., class c2 columns] ----
  P.sW2.nsplit = true;
  for (auto& zb : P.zbase) {
    const int b2 = zb.first.first, mpp = zb.first.second;
    const ColLayout& zl = collayout(r.sub(th.mq[mpp], H.bq[b2]));
    for (int co = 0; co < ncls; ++co) {
      if (zl.off[co] < 0) continue;
      const int64_t cd = zl.dim[co];
      GemmTask t{};
      t.c_off = zb.second + zl.off[co];
      t.m = (int32_t)H.cls_mem[co].size();
      t.n = (int32_t)(th.nrows[mpp] * cd);
      t.ldc = (int32_t)cd;
      t.n_in = (int32_t)cd;
      t.ldc_out = (int32_t)zl.n;
      t.t0 = (int32_t)P.sW2.terms.size();
      for (auto& kv : P.opoff) {
        if (kv.first[1] != b2 || kv.first[3] != co) continue;
        const int b1 = kv.first[0], ci = kv.first[2];
        const int m = th.find(r.sub(th.mq[mpp], H.bq[b1]));
        if (m < 0 || ccoff[m][ci] < 0) continue;
        auto yb = P.ybase.find({b1, m});
        if (yb == P.ybase.end()) continue;
        if (ccdim[m][ci] != cd) return fail(CMPS_ERR_STATE, "canonical order: W2 sector mismatch");
        GemmTerm tm{};
        tm.a_off = kv.second;
        tm.lda = (int32_t)H.cls_mem[ci].size();
        tm.k = (int32_t)H.cls_mem[ci].size();
        tm.b_off = yb->second + ccoff[m][ci];
        tm.ldb = (int32_t)cd;
        tm.ldb_out = (int32_t)th.ncols[m];
        P.sW2.terms.push_back(tm);
        P.flops += term_flops(t, tm);
      }
      t.t1 = (int32_t)P.sW2.terms.size();
      P.sW2.tasks.push_back(t);
    }
  }
  // ---- stage R: Theta'_m''[., s2'] = sum_b2 Z^{b2}_m''[., s2' columns] . R^{b2} ----
  for (int mpp = 0; mpp < nm; ++mpp) {
    if (!H.owned[mpp]) continue;
    for (int c = 0; c < ncls; ++c) {
      if (ccoff[mpp][c] < 0) continue;
      const int tp = A2.find(r.add(th.mq[mpp], H.sigq[H.cls_mem[c][0]]));  // a2' sector
      for (size_t i = 0; i < H.cls_mem[c].size(); ++i) {
        GemmTask t{};
        if (H.out_base[mpp] < 0) return fail(CMPS_ERR_ARG, "output window lacks an owned sector");
        t.c_off = H.out_base[mpp] + ccoff[mpp][c] + (int64_t)i * ccdim[mpp][c];
        t.m = (int32_t)th.nrows[mpp];
        t.n = (int32_t)A2.sdim[tp];
        t.ldc = (int32_t)th.ncols[mpp];
        t.t0 = (int32_t)P.sR.terms.size();
        for (int b2 : br_used) {
          auto zb = P.zbase.find({b2, mpp});
          if (zb == P.zbase.end()) continue;
          const QKey mu = r.sub(th.mq[mpp], H.bq[b2]);
          const ColLayout& zl = collayout(mu);
          if (zl.off[c] < 0) continue;
          const int ta = A2.find(r.add(mu, H.sigq[H.cls_mem[c][0]]));  // a2 sector
          const int64_t ro = H.R.off[(size_t)b2 * ns2 + ta];
          if (ro < 0 || H.R.partner[(size_t)b2 * ns2 + ta] != tp) continue;
          GemmTerm tm{};
          tm.a_off = zb->second + zl.off[c] + (int64_t)i * zl.dim[c];
          tm.lda = (int32_t)zl.n;
          tm.k = (int32_t)A2.sdim[ta];
          tm.b_off = ro;  // R^{b2} stored [a2][a2']
          tm.ldb = (int32_t)A2.sdim[tp];
          P.sR.terms.push_back(tm);
          P.flops += term_flops(t, tm);
        }
        t.t1 = (int32_t)P.sR.terms.size();
        P.sR.tasks.push_back(t);
      }
    }
  }
  return CMPS_OK;
}

int canonical_scratch(const Heff& H, const Planar** xz, const Planar** y) {
  if (!H.canon) return fail(CMPS_ERR_STATE, "canonical-order plans not built");
  *xz = &H.canon->xz;
  *y = &H.canon->y;
  return CMPS_OK;
}

int canonical_flops(const Heff& H, double* flops, std::vector<uint8_t>* need) {
  Plan P;
  CMPS_TRY(plan_canonical(H, P));
  *flops = P.flops;
  if (need) {
    *need = P.need;
    need->resize(H.th.mq.size(), 0);
  }
  return CMPS_OK;
}

int build_canonical(Heff& H) {
  release_canonical(&H);
  Plan P;
  CMPS_TRY(plan_canonical(H, P));
  if (P.missing) return fail(CMPS_ERR_ARG, "input window lacks a sector the owned outputs read");
  auto* C = new (std::nothrow) Canon();
  if (!C) return fail(CMPS_ERR_NOMEM, "host allocation failed");
  H.canon = C;
  cudaStream_t st = H.ctx->stream;
  auto bail = [&](int rc) {
    release_canonical(&H);
    return rc;
  };
  int rc;
  if ((rc = C->ops.alloc(std::max<int64_t>(P.ops_len, 1))) != CMPS_OK) return bail(rc);
  if ((rc = copy_wait(C->ops.re(), P.ops_re.data(), sizeof(double) * P.ops_len, cudaMemcpyHostToDevice, st)) !=
      CMPS_OK)
    return bail(rc);
  if ((rc = copy_wait(C->ops.im(), P.ops_im.data(), sizeof(double) * P.ops_len, cudaMemcpyHostToDevice, st)) !=
      CMPS_OK)
    return bail(rc);
  const int64_t xz = std::max<int64_t>(std::max(P.x_len, P.z_len), 1);
  if ((rc = C->xz.alloc(xz)) != CMPS_OK) return bail(rc);
  if ((rc = C->y.alloc(std::max<int64_t>(P.y_len, 1))) != CMPS_OK) return bail(rc);
  // every operand and output range inside its buffer, before any launch
  if ((rc = P.sL.validate(false, false, H.L.data.len, H.in_len, xz, "canonical stage L")) != CMPS_OK ||
      (rc = P.sW1.validate(false, false, C->ops.len, xz, C->y.len, "canonical stage W1")) != CMPS_OK ||
      (rc = P.sW2.validate(false, false, C->ops.len, C->y.len, xz, "canonical stage W2")) != CMPS_OK ||
      (rc = P.sR.validate(false, false, xz, H.R.data.len, H.out_len, "canonical stage R")) != CMPS_OK)
    return bail(rc);
  C->sL = std::move(P.sL);
  C->sW1 = std::move(P.sW1);
  C->sW2 = std::move(P.sW2);
  C->sR = std::move(P.sR);
  for (GemmPlan* p : {&C->sL, &C->sW1, &C->sW2, &C->sR})
    if ((rc = p->upload(st)) != CMPS_OK) return bail(rc);
  C->flops = P.flops;
  return CMPS_OK;
}

int build_canonical32(Heff& H) {
  Canon* C = H.canon;
  if (!C) return fail(CMPS_ERR_STATE, "canonical-order plans not built");
  if (C->have32) return CMPS_OK;
  cudaStream_t st = H.ctx->stream;
  CMPS_TRY(C->ops32.alloc(C->ops.len));
  CMPS_TRY(C->L32.alloc(H.L.data.len));
  CMPS_TRY(C->R32.alloc(H.R.data.len));
  CMPS_TRY(C->x32.alloc(std::max<int64_t>(1, H.in_len)));
  CMPS_TRY(C->o32.alloc(std::max<int64_t>(1, H.out_len)));
  CMPS_TRY(to_fp32(C->ops.re(), C->ops.im(), C->ops.len, C->ops32, st));
  CMPS_TRY(to_fp32(H.L.data.re(), H.L.data.im(), H.L.data.len, C->L32, st));
  CMPS_TRY(to_fp32(H.R.data.re(), H.R.data.im(), H.R.data.len, C->R32, st));
  C->xz32.d = (float*)C->xz.d;  // 2 len floats inside 2 len doubles
  C->xz32.len = C->xz.len;
  C->y32.d = (float*)C->y.d;
  C->y32.len = C->y.len;
  CMPS_CUDA(cudaStreamSynchronize(st));
  C->have32 = true;
  return CMPS_OK;
}

// The low-precision canonical matvec: theta (FP64) -> FP32, the four stages
// on FP32 planes with FP32 accumulation, the owned output sectors -> FP64.
int apply_canonical32(Heff& H, int which, const Planar& in, Planar& out, cudaStream_t st) {
  Canon* C = H.canon;
  if (!C || !C->have32) return fail(CMPS_ERR_STATE, "canonical-order FP32 operands not prepared");
  if (which != 2) {
    CMPS_TRY(to_fp32(in.re(), in.im(), H.in_len, C->x32, st));
    CMPS_TRY(launch_cgemm_fp32(C->sL, C->L32, C->x32, C->xz32, st));
    CMPS_TRY(launch_cgemm_fp32(C->sW1, C->ops32, C->xz32, C->y32, st));
  }
  if (which != 1) {
    CMPS_TRY(launch_cgemm_fp32(C->sW2, C->ops32, C->y32, C->xz32, st));
    CMPS_TRY(launch_cgemm_fp32(C->sR, C->xz32, C->R32, C->o32, st));
    if (H.all_owned()) {
      CMPS_TRY(to_fp64(C->o32, H.out_len, out.re(), out.im(), st));
    } else {
      // sharded: only the owned sectors were computed; the others stay unwritten
      Planar32 v;
      for (size_t m = 0; m < H.th.mq.size(); ++m) {
        if (!H.owned[m]) continue;
        const int64_t off = H.out_base[m], n = H.th.nrows[m] * H.th.ncols[m];
        v.d = C->o32.d + off;
        v.len = C->o32.len;  // plane stride of o32
        CMPS_TRY(to_fp64(v, n, out.re() + off, out.im() + off, st));
      }
      v.d = nullptr;
    }
  }
  return CMPS_OK;
}

// The four canonical plans' tile shapes, measured (autotune_plan): on the FP32
// operands when the handle runs the FP32 form, else on the FP64 ones.  The
// input is the handle's zeroed work vector, the output its other one.
int autotune_canonical(Heff& H, bool fp32, cudaStream_t st, TuneStats* stats) {
  Canon* C = H.canon;
  if (!C) return CMPS_OK;
  Planar in, out;
  in.d = H.x.d;
  in.len = H.in_len;
  out.d = H.y.d;
  out.len = H.out_len;
  int rc = CMPS_OK;
  if (fp32) {
    if (!C->have32) rc = fail(CMPS_ERR_STATE, "canonical-order FP32 operands not prepared");
    if (rc == CMPS_OK) rc = to_fp32(in.re(), in.im(), H.in_len, C->x32, st);
    if (rc == CMPS_OK) rc = autotune_plan(C->sL, 20, [&] { return launch_cgemm_fp32(C->sL, C->L32, C->x32, C->xz32, st); }, st, stats);
    if (rc == CMPS_OK) rc = autotune_plan(C->sW1, 21, [&] { return launch_cgemm_fp32(C->sW1, C->ops32, C->xz32, C->y32, st); }, st, stats);
    if (rc == CMPS_OK) rc = autotune_plan(C->sW2, 22, [&] { return launch_cgemm_fp32(C->sW2, C->ops32, C->y32, C->xz32, st); }, st, stats);
    if (rc == CMPS_OK) rc = autotune_plan(C->sR, 23, [&] { return launch_cgemm_fp32(C->sR, C->xz32, C->R32, C->o32, st); }, st, stats);
  } else {
    rc = autotune_plan(C->sL, 10, [&] { return launch_zgemm_fp64(C->sL, false, false, H.L.data, in, C->xz, st); }, st, stats);
    if (rc == CMPS_OK) rc = autotune_plan(C->sW1, 11, [&] { return launch_zgemm_fp64(C->sW1, false, false, C->ops, C->xz, C->y, st); }, st, stats);
    if (rc == CMPS_OK) rc = autotune_plan(C->sW2, 12, [&] { return launch_zgemm_fp64(C->sW2, false, false, C->ops, C->y, C->xz, st); }, st, stats);
    if (rc == CMPS_OK) rc = autotune_plan(C->sR, 13, [&] { return launch_zgemm_fp64(C->sR, false, false, C->xz, H.R.data, out, st); }, st, stats);
  }
  in.d = out.d = nullptr;
  return rc;
}

// which: 1 = stages L and W1, 2 = stages W2 and R, 0 = all four.
int apply_canonical(Heff& H, int which, const Planar& in, Planar& out, cudaStream_t st) {
  Canon* C = H.canon;
  if (!C) return fail(CMPS_ERR_STATE, "canonical-order plans not built");
  if (which != 2) {
    CMPS_TRY(launch_zgemm_fp64(C->sL, false, false, H.L.data, in, C->xz, st));
    CMPS_TRY(launch_zgemm_fp64(C->sW1, false, false, C->ops, C->xz, C->y, st));
  }
  if (which != 1) {
    CMPS_TRY(launch_zgemm_fp64(C->sW2, false, false, C->ops, C->y, C->xz, st));
    CMPS_TRY(launch_zgemm_fp64(C->sR, false, false, C->xz, H.R.data, out, st));
  }
  return CMPS_OK;
}

}  // namespace cmps
