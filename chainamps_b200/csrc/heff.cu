// Host side of the device-resident effective Hamiltonian: parsing of the
// reference's MPX tensors, charge-sector structure, LeftPart / RightPart
// formation, the two grouped-GEMM stages of the matvec and the Krylov
// ground-state solver.
//
// Matvec (TwoVertexMPOMPSMultiply, DMRG_routines.cpp:898-945):
//   LeftPart^{b1}[(s1', a0'), (s1, a0)]  = sum_b0 W[s1', b0, s1, b1] L^{b0}[a0', a0]
//   RightPart^{b1}[(s2, a2), (s2', a2')] = sum_b2 W[s2', b1, s2, b2] R^{b2}[a2', a2]
//   T^{b1}  = LeftPart^{b1} . Theta                       (stage 1)
//   Theta'  = sum_b1 T^{b1} . RightPart^{b1}               (stage 2)
// exactly the reference's (LeftPart . V) . RightPart order
// (DMRG_routines.cpp:779, :943), with every operand held as dense
// charge-sector blocks instead of CSC.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <numeric>
#include <set>

#include "heff.h"

namespace cmps {

// ---------------------------------------------------------------------------
QKey Rules::add(const QKey& a, const QKey& b) const {
  QKey o = zero();
  for (int i = 0; i < nq; ++i) {
    int v = (int)a[i] + (int)b[i];
    if (n[i] > 0) v = ((v % n[i]) + n[i]) % n[i];
    o[i] = (int16_t)v;
  }
  return o;
}
QKey Rules::sub(const QKey& a, const QKey& b) const {
  QKey o = zero();
  for (int i = 0; i < nq; ++i) {
    int v = (int)a[i] - (int)b[i];
    if (n[i] > 0) v = ((v % n[i]) + n[i]) % n[i];
    o[i] = (int16_t)v;
  }
  return o;
}

void Bond::build(const std::vector<QKey>& charges) {
  sq.clear(); sdim.clear(); esec.assign(charges.size(), 0); epos.assign(charges.size(), 0);
  selem.clear(); lookup.clear();
  for (size_t e = 0; e < charges.size(); ++e) {
    auto it = lookup.find(charges[e]);
    int s;
    if (it == lookup.end()) {
      s = (int)sq.size();
      lookup[charges[e]] = s;
      sq.push_back(charges[e]);
      sdim.push_back(0);
      selem.emplace_back();
    } else {
      s = it->second;
    }
    esec[e] = s;
    epos[e] = sdim[s]++;
    selem[s].push_back((int64_t)e);
  }
}

std::vector<QKey> Bond::element_charges() const {
  std::vector<QKey> out(esec.size());
  for (size_t e = 0; e < esec.size(); ++e) out[e] = sq[esec[e]];
  return out;
}

int Planar::alloc(int64_t n) {
  release();
  len = n;
  if (n == 0) return CMPS_OK;
  cudaError_t e = dmalloc(&d, sizeof(double) * 2 * (size_t)n);
  if (e != cudaSuccess) {
    d = nullptr;
    len = 0;
    return fail(CMPS_ERR_NOMEM, std::string("device allocation of ") + std::to_string(16.0 * n / 1e9) +
                                    " GB failed: " + cudaGetErrorString(e));
  }
  return CMPS_OK;
}

void Planar::release() {
  if (d) dfree(d);
  d = nullptr;
  len = 0;
}

int64_t Env::block_rows(int b, int s) const {
  int sp = partner[(size_t)b * a.nsec() + s];
  return right ? a.sdim[s] : a.sdim[sp];
}
int64_t Env::block_cols(int b, int s) const {
  int sp = partner[(size_t)b * a.nsec() + s];
  return right ? a.sdim[sp] : a.sdim[s];
}

// ---------------------------------------------------------------------------
// desc helpers
static int check_desc(const cmps_mpx_desc* d, int nidx, const char* what) {
  if (!d) return fail(CMPS_ERR_ARG, std::string(what) + ": null descriptor");
  if (d->num_indices != nidx)
    return fail(CMPS_ERR_ARG, std::string(what) + ": expected " + std::to_string(nidx) + " indices, got " +
                                  std::to_string(d->num_indices));
  if (d->num_row_indices < 0 || d->num_row_indices > d->num_indices)
    return fail(CMPS_ERR_ARG, std::string(what) + ": bad num_row_indices");
  int64_t r = 1, c = 1;
  for (int i = 0; i < d->num_indices; ++i) {
    if (d->sizes[i] < 1) return fail(CMPS_ERR_ARG, std::string(what) + ": empty index");
    (i < d->num_row_indices ? r : c) *= d->sizes[i];
  }
  if (r != d->rows || c != d->cols)
    return fail(CMPS_ERR_ARG, std::string(what) + ": matrix shape does not match index sizes");
  if (d->colptr[0] != 0) return fail(CMPS_ERR_ARG, std::string(what) + ": colptr[0] != 0");
  for (int64_t j = 0; j < d->cols; ++j)
    if (d->colptr[j + 1] < d->colptr[j]) return fail(CMPS_ERR_ARG, std::string(what) + ": colptr not monotone");
  int64_t nnz = d->colptr[d->cols];
  for (int64_t p = 0; p < nnz; ++p)
    if (d->rowind[p] < 0 || d->rowind[p] >= d->rows)
      return fail(CMPS_ERR_ARG, std::string(what) + ": row index out of range");
  return CMPS_OK;
}

int parse_index_charges(const Rules& r, const cmps_mpx_desc* d, int idx, std::vector<QKey>& out) {
  int64_t off = 0;
  for (int i = 0; i < idx; ++i) off += d->sizes[i];
  out.assign(d->sizes[idx], r.zero());
  for (int64_t e = 0; e < d->sizes[idx]; ++e) {
    QKey q = r.zero();
    for (int c = 0; c < r.nq; ++c) {
      int v = d->charges[(off + e) * r.nq + c];
      if (r.n[c] > 0) v = ((v % r.n[c]) + r.n[c]) % r.n[c];
      q[c] = (int16_t)v;
    }
    out[e] = q;
  }
  return CMPS_OK;
}

// Visit every stored entry with its multi-index (first index fastest).
template <typename F>
static void for_each_entry(const cmps_mpx_desc* d, F&& f) {
  int k = d->num_indices, nr = d->num_row_indices;
  std::vector<int64_t> mi(k, 0);
  for (int64_t c = 0; c < d->cols; ++c) {
    int64_t cc = c;
    for (int i = nr; i < k; ++i) {
      mi[i] = cc % d->sizes[i];
      cc /= d->sizes[i];
    }
    for (int64_t p = d->colptr[c]; p < d->colptr[c + 1]; ++p) {
      int64_t rr = d->rowind[p];
      for (int i = 0; i < nr; ++i) {
        mi[i] = rr % d->sizes[i];
        rr /= d->sizes[i];
      }
      f(mi.data(), d->values[2 * p], d->values[2 * p + 1]);
    }
  }
}

// L: a' = 1, b = 3, a = 5.  R: a' = 0, b = 2, a = 4.  Blocks are allocated
// for every (b, sector) with a charge-consistent partner sector.
int build_env_from_desc(const Rules& r, const cmps_mpx_desc* d, bool right, Env& env, int D,
                        const std::vector<QKey>& bq, cudaStream_t st) {
  const char* what = right ? "right block" : "left block";
  CMPS_TRY(check_desc(d, 6, what));
  const int ia = right ? 4 : 5, iap = right ? 0 : 1, ib = right ? 2 : 3;
  for (int i = 0; i < 6; ++i)
    if (i != ia && i != iap && i != ib && d->sizes[i] != 1)
      return fail(CMPS_ERR_ARG, std::string(what) + ": index " + std::to_string(i) + " must be a size-1 dummy");
  if (d->sizes[ib] != D) return fail(CMPS_ERR_ARG, std::string(what) + ": MPO index size differs from W");
  std::vector<QKey> qa, qap, qb;
  parse_index_charges(r, d, ia, qa);
  parse_index_charges(r, d, iap, qap);
  parse_index_charges(r, d, ib, qb);
  if (qa.size() != qap.size() || qa != qap)
    return fail(CMPS_ERR_ARG, std::string(what) + ": bra and ket bond indices differ");
  if (qb != bq) return fail(CMPS_ERR_ARG, std::string(what) + ": MPO index charges differ from W");
  env.right = right;
  env.a.build(qa);
  env.D = D;
  env.bq = bq;
  const int ns = env.a.nsec();
  env.off.assign((size_t)D * ns, -1);
  env.partner.assign((size_t)D * ns, -1);
  int64_t total = 0;
  for (int b = 0; b < D; ++b)
    for (int s = 0; s < ns; ++s) {
      int sp = env.a.find(r.add(env.a.sq[s], bq[b]));
      if (sp < 0) continue;
      env.partner[(size_t)b * ns + s] = sp;
      env.off[(size_t)b * ns + s] = total;
      total += env.a.sdim[s] * env.a.sdim[sp];
    }
  std::vector<double> h(2 * (size_t)total, 0.0);
  int status = CMPS_OK;
  for_each_entry(d, [&](const int64_t* mi, double re, double im) {
    if (status != CMPS_OK) return;
    int64_t a = mi[ia], ap = mi[iap], b = mi[ib];
    int s = env.a.esec[a], sp = env.a.esec[ap];
    if (env.partner[(size_t)b * ns + s] != sp) {
      if (re != 0.0 || im != 0.0) status = fail(CMPS_ERR_CHARGE, std::string(what) + ": entry violates charge conservation");
      return;
    }
    int64_t o = env.off[(size_t)b * ns + s];
    int64_t p = env.a.epos[a], pp = env.a.epos[ap];
    int64_t e = right ? o + p * env.a.sdim[sp] + pp : o + pp * env.a.sdim[s] + p;
    h[e] += re;
    h[total + e] += im;
  });
  if (status != CMPS_OK) return status;
  CMPS_TRY(env.data.alloc(total));
  CMPS_TRY(copy_wait(env.data.d, h.data(), sizeof(double) * 2 * total, cudaMemcpyHostToDevice, st));
  return CMPS_OK;
}

// ---------------------------------------------------------------------------
Heff::~Heff() {
  release_split(this);
  release_canonical(this);
  L.data.release();
  R.data.release();
  LP.release();
  RP.release();
  T.release();
  x.release();
  y.release();
  theta.release();
  kv.release();
  proj.release();
  if (d_proj) dfree(d_proj);
  d_proj = nullptr;
  stage1.release();
  stage2.release();
  ops.release();
  if (d_pack) dfree(d_pack);
  if (d_io) dfree(d_io);
  if (h_ab) cudaFreeHost(h_ab);
  if (d_lp_blocks) dfree(d_lp_blocks);
  if (d_lp_terms) dfree(d_lp_terms);
  if (d_rp_blocks) dfree(d_rp_blocks);
  if (d_rp_terms) dfree(d_rp_terms);
}

template <typename T>
static int upload_vec(const std::vector<T>& v, T** d, cudaStream_t st) {
  if (*d) dfree(*d);
  *d = nullptr;
  if (v.empty()) return CMPS_OK;
  CMPS_CUDA(dmalloc((void**)d, sizeof(T) * v.size()));
  return copy_wait(*d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, st);
}

int Heff::build(cmps_context* c, const Rules& r, const cmps_mpx_desc* Ld, const cmps_mpx_desc* Wd,
                const cmps_mpx_desc* Rd) {
  ctx = c;
  device = c->device;
  rules = r;
  CMPS_TRY(parse_mpo(Wd));
  CMPS_TRY(build_env_from_desc(r, Ld, false, L, D, bq, c->stream));
  CMPS_TRY(build_env_from_desc(r, Rd, true, R, D, bq, c->stream));
  return finish();
}

int copy_env(const Env& src, Env& dst, cudaStream_t st) {
  dst.a = src.a;
  dst.D = src.D;
  dst.bq = src.bq;
  dst.off = src.off;
  dst.partner = src.partner;
  dst.right = src.right;
  CMPS_TRY(dst.data.alloc(src.data.len));
  CMPS_TRY(copy_wait(dst.data.d, src.data.d, sizeof(double) * 2 * src.data.len, cudaMemcpyDeviceToDevice, st));
  return CMPS_OK;
}

int Heff::build_from_envs(cmps_context* c, const Rules& r, const Env& Lsrc, const cmps_mpx_desc* Wd,
                          const Env& Rsrc) {
  ctx = c;
  device = c->device;
  rules = r;
  CMPS_TRY(parse_mpo(Wd));
  if (Lsrc.right || !Rsrc.right) return fail(CMPS_ERR_ARG, "block handedness: need a left and a right block");
  if (Lsrc.D != D || Rsrc.D != D || Lsrc.bq != bq || Rsrc.bq != bq)
    return fail(CMPS_ERR_ARG, "block MPO index differs from W");
  CMPS_TRY(copy_env(Lsrc, L, c->stream));
  CMPS_TRY(copy_env(Rsrc, R, c->stream));
  return finish();
}

int Heff::parse_mpo(const cmps_mpx_desc* Wd) {
  const Rules& r = rules;
  CMPS_TRY(check_desc(Wd, 4, "MPO"));
  d = (int)Wd->sizes[0];
  D = (int)Wd->sizes[1];
  if (Wd->sizes[2] != d || Wd->sizes[3] != D) return fail(CMPS_ERR_ARG, "MPO: index sizes inconsistent");
  std::vector<QKey> sig2, bq3;
  parse_index_charges(r, Wd, 0, sigq);
  parse_index_charges(r, Wd, 2, sig2);
  parse_index_charges(r, Wd, 1, bq);
  parse_index_charges(r, Wd, 3, bq3);
  if (sigq != sig2 || bq != bq3) return fail(CMPS_ERR_ARG, "MPO: row and column index charges differ");
  W.clear();
  int status = CMPS_OK;
  for_each_entry(Wd, [&](const int64_t* mi, double re, double im) {
    if (re == 0.0 && im == 0.0) return;
    int sp = (int)mi[0], bl = (int)mi[1], s = (int)mi[2], br = (int)mi[3];
    if (r.add(sigq[sp], bq[bl]) != r.add(sigq[s], bq[br])) {
      status = fail(CMPS_ERR_CHARGE, "MPO: entry violates charge conservation");
      return;
    }
    W.push_back(WEntry{sp, bl, s, br, re, im});
  });
  if (status != CMPS_OK) return status;
  return CMPS_OK;
}

// One CTA per ARPACK column: out[start + i] for the i-th allowed row of the
// column's sector block (mode 0: theta offset, mode 1: full linear index).
__global__ void k_arpack_map(const Heff::MapCol* __restrict__ cols, const Heff::MapSec* __restrict__ secs,
                             const int64_t* __restrict__ rowlin, const int64_t* __restrict__ rowth, int64_t dchiL,
                             int mode, int64_t* __restrict__ out) {
  const Heff::MapCol c = cols[blockIdx.x];
  const Heff::MapSec s = secs[c.m];
  for (int64_t i = threadIdx.x; i < s.nrows; i += blockDim.x) {
    const int64_t r = s.rowstart + i;
    out[c.start + i] = mode == 0 ? s.base + rowth[r] * s.ncols + c.colth : rowlin[r] + dchiL * c.colpart;
  }
}

int Heff::arpack_map(int mode, int64_t* d_out, cudaStream_t st) const {
  if (map_cols.empty() || n_allowed == 0) return CMPS_OK;
  if (map_cols.size() > 0x7fffffffull) return fail(CMPS_ERR_ARG, "too many wavefunction columns");
  MapCol* dc = nullptr;
  MapSec* ds = nullptr;
  int64_t *drl = nullptr, *drt = nullptr;
  int rc = CMPS_OK;
  auto up = [&](auto& v, auto** d) -> int {
    const size_t bytes = sizeof(v[0]) * std::max<size_t>(1, v.size());
    CMPS_CUDA(dmalloc((void**)d, bytes));
    return copy_wait(*d, v.data(), sizeof(v[0]) * v.size(), cudaMemcpyHostToDevice, st);
  };
  if ((rc = up(map_cols, &dc)) == CMPS_OK && (rc = up(map_secs, &ds)) == CMPS_OK &&
      (rc = up(map_rowlin, &drl)) == CMPS_OK && (rc = up(map_rowth, &drt)) == CMPS_OK) {
    const int64_t dchiL = (int64_t)d * L.a.size();
    k_arpack_map<<<(unsigned)map_cols.size(), 256, 0, st>>>(dc, ds, drl, drt, dchiL, mode, d_out);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = fail(CMPS_ERR_CUDA, std::string("ARPACK index map: ") + cudaGetErrorString(e));
  }
  if (dc) dfree(dc);
  if (ds) dfree(ds);
  if (drl) dfree(drl);
  if (drt) dfree(drt);
  return rc;
}

int Heff::allowed_indices(int64_t* host_out) const {
  if (n_allowed == 0) return CMPS_OK;
  int64_t* tmp = nullptr;
  CMPS_CUDA(dmalloc(&tmp, sizeof(int64_t) * n_allowed));
  int rc = arpack_map(1, tmp, ctx->stream);
  if (rc == CMPS_OK) rc = copy_wait(host_out, tmp, sizeof(int64_t) * n_allowed, cudaMemcpyDeviceToHost, ctx->stream);
  dfree(tmp);
  return rc;
}

// ARPACK order -> sector blocks: CTA = (group of <= 32 columns, 32 rows).
// Reads run down each ARPACK column (contiguous), writes along theta rows
// (the group's columns are consecutive theta columns).
template <bool PACK>
__global__ void __launch_bounds__(256) k_pack_tiles(const Heff::PackTile* __restrict__ tiles,
                                                    const Heff::PackGroup* __restrict__ groups,
                                                    const int32_t* __restrict__ gcols,
                                                    const Heff::MapCol* __restrict__ cols,
                                                    const Heff::MapSec* __restrict__ secs,
                                                    const int64_t* __restrict__ rowth, double2* __restrict__ arp,
                                                    double* __restrict__ re, double* __restrict__ im) {
  __shared__ double2 t[32][33];  // [column j][row r]
  const Heff::PackTile tl = tiles[blockIdx.x];
  const Heff::PackGroup g = groups[tl.group];
  const Heff::MapSec s = secs[g.m];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int64_t left = s.nrows - tl.r0;
  const int nr = left < 32 ? (int)left : 32;
  if (PACK) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int j = ty + 8 * k, r = tx;
      if (j < g.cnt && r < nr) t[j][r] = arp[cols[gcols[g.off + j]].start + tl.r0 + r];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int r = ty + 8 * k, j = tx;
      if (j < g.cnt && r < nr) {
        const int64_t p = s.base + rowth[s.rowstart + tl.r0 + r] * s.ncols + cols[gcols[g.off + j]].colth;
        const double2 v = t[j][r];
        re[p] = v.x;
        im[p] = v.y;
      }
    }
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int r = ty + 8 * k, j = tx;
      if (j < g.cnt && r < nr) {
        const int64_t p = s.base + rowth[s.rowstart + tl.r0 + r] * s.ncols + cols[gcols[g.off + j]].colth;
        t[j][r] = make_double2(re[p], im[p]);
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int j = ty + 8 * k, r = tx;
      if (j < g.cnt && r < nr) arp[cols[gcols[g.off + j]].start + tl.r0 + r] = t[j][r];
    }
  }
}

int Heff::build_pack(cudaStream_t st) {
  // ARPACK column index of (a2, s2), then groups per (m, s2) in a2-sector order
  const Bond& A2 = R.a;
  std::vector<int32_t> col_of((size_t)A2.size() * d, -1);
  for (size_t c = 0; c < map_cols.size(); ++c) {
    const int64_t s2 = map_cols[c].colpart % d, a2 = map_cols[c].colpart / d;
    col_of[(size_t)a2 * d + s2] = (int32_t)c;
  }
  std::vector<std::vector<int64_t>> elems(A2.nsec());
  for (int64_t a2 = 0; a2 < A2.size(); ++a2) elems[A2.esec[a2]].push_back(a2);
  std::vector<int32_t> gcols;
  std::vector<PackGroup> groups;
  std::vector<PackTile> tiles;
  for (int m = 0; m < (int)th.mq.size(); ++m)
    for (int s2 = 0; s2 < d; ++s2) {
      if (th.coloff[m][s2] < 0) continue;
      const int t = A2.find(rules.add(th.mq[m], sigq[s2]));
      const std::vector<int64_t>& el = elems[t];
      for (size_t e0 = 0; e0 < el.size(); e0 += 32) {
        PackGroup g{(int64_t)gcols.size(), (int32_t)std::min<size_t>(32, el.size() - e0), m};
        for (int j = 0; j < g.cnt; ++j) {
          const int32_t c = col_of[(size_t)el[e0 + j] * d + s2];
          if (c < 0 || map_cols[c].m != m || map_cols[c].colth != th.coloff[m][s2] + (int64_t)(e0 + j))
            return fail(CMPS_ERR_STATE, "internal: pack group columns not consecutive");
          gcols.push_back(c);
        }
        for (int64_t r0 = 0; r0 < th.nrows[m]; r0 += 32) tiles.push_back(PackTile{(int32_t)groups.size(), (int32_t)r0});
        groups.push_back(g);
      }
    }
  if (tiles.size() > 0x7fffffffull) return fail(CMPS_ERR_ARG, "too many pack tiles");
  n_pack_tiles = 0;
  if (tiles.empty()) return CMPS_OK;
  auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
  const size_t b_cols = al(sizeof(MapCol) * map_cols.size()), b_secs = al(sizeof(MapSec) * map_secs.size()),
               b_rowth = al(sizeof(int64_t) * map_rowth.size()), b_gcols = al(sizeof(int32_t) * gcols.size()),
               b_groups = al(sizeof(PackGroup) * groups.size()), b_tiles = al(sizeof(PackTile) * tiles.size());
  if (d_pack) dfree(d_pack);
  d_pack = nullptr;
  CMPS_CUDA(dmalloc(&d_pack, b_cols + b_secs + b_rowth + b_gcols + b_groups + b_tiles));
  char* p = (char*)d_pack;
  d_map_cols = (const MapCol*)p;
  CMPS_TRY(copy_wait(p, map_cols.data(), sizeof(MapCol) * map_cols.size(), cudaMemcpyHostToDevice, st));
  p += b_cols;
  d_map_secs = (const MapSec*)p;
  CMPS_TRY(copy_wait(p, map_secs.data(), sizeof(MapSec) * map_secs.size(), cudaMemcpyHostToDevice, st));
  p += b_secs;
  d_map_rowth = (const int64_t*)p;
  CMPS_TRY(copy_wait(p, map_rowth.data(), sizeof(int64_t) * map_rowth.size(), cudaMemcpyHostToDevice, st));
  p += b_rowth;
  d_pack_gcols = (const int32_t*)p;
  CMPS_TRY(copy_wait(p, gcols.data(), sizeof(int32_t) * gcols.size(), cudaMemcpyHostToDevice, st));
  p += b_gcols;
  d_pack_groups = (const PackGroup*)p;
  CMPS_TRY(copy_wait(p, groups.data(), sizeof(PackGroup) * groups.size(), cudaMemcpyHostToDevice, st));
  p += b_groups;
  d_pack_tiles = (const PackTile*)p;
  CMPS_TRY(copy_wait(p, tiles.data(), sizeof(PackTile) * tiles.size(), cudaMemcpyHostToDevice, st));
  n_pack_tiles = (int64_t)tiles.size();
  return CMPS_OK;
}

int Heff::pack(const double* in, const Planar& out, cudaStream_t st) const {
  if (n_pack_tiles == 0) return CMPS_OK;
  k_pack_tiles<true><<<(unsigned)n_pack_tiles, 256, 0, st>>>(d_pack_tiles, d_pack_groups, d_pack_gcols, d_map_cols,
                                                             d_map_secs, d_map_rowth, (double2*)in, out.re(), out.im());
  CMPS_CUDA(cudaGetLastError());
  return CMPS_OK;
}

int Heff::unpack(const Planar& in, double* out, cudaStream_t st) const {
  if (n_pack_tiles == 0) return CMPS_OK;
  k_pack_tiles<false><<<(unsigned)n_pack_tiles, 256, 0, st>>>(d_pack_tiles, d_pack_groups, d_pack_gcols, d_map_cols,
                                                              d_map_secs, d_map_rowth, (double2*)out, in.re(), in.im());
  CMPS_CUDA(cudaGetLastError());
  return CMPS_OK;
}

// Phase timer of Heff::finish for CMPS_BUILD_TRACE (host wall ms to stderr).
struct BuildTrace {
  bool on = std::getenv("CMPS_BUILD_TRACE") != nullptr;
  std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
  void mark(const char* what) {
    if (!on) return;
    const auto now = std::chrono::steady_clock::now();
    std::fprintf(stderr, "build %-22s %8.2f ms\n", what, std::chrono::duration<double, std::milli>(now - t).count());
    t = now;
  }
};

int Heff::finish() {
  BuildTrace bt;
  const Rules& r = rules;
  const Bond& A0 = L.a;
  const Bond& A2 = R.a;
  // ---- theta space ----
  // middle charges ordered by first appearance over columns c = s2 + d*a2
  // ascending (the block order of GetAllBlockColumns, MPX_matrix.cpp:365-385)
  std::set<QKey> rowm;
  for (int s1 = 0; s1 < d; ++s1)
    for (int s = 0; s < A0.nsec(); ++s) rowm.insert(r.add(sigq[s1], A0.sq[s]));
  th = ThetaSpace();
  for (int64_t a2 = 0; a2 < A2.size(); ++a2)
    for (int s2 = 0; s2 < d; ++s2) {
      QKey m = r.sub(A2.sq[A2.esec[a2]], sigq[s2]);
      if (!rowm.count(m) || th.mfind.count(m)) continue;
      th.mfind[m] = (int)th.mq.size();
      th.mq.push_back(m);
    }
  const int nm = (int)th.mq.size();
  // charge classes of the physical states; blocks list states class by class
  cls_mem.clear();
  cls_of.assign(d, -1);
  cls_pos.assign(d, -1);
  {
    std::map<QKey, int> cfind;
    for (int s = 0; s < d; ++s) {
      auto it = cfind.find(sigq[s]);
      int c = it == cfind.end() ? -1 : it->second;
      if (c < 0) {
        c = (int)cls_mem.size();
        cfind[sigq[s]] = c;
        cls_mem.emplace_back();
      }
      cls_of[s] = c;
      cls_pos[s] = (int)cls_mem[c].size();
      cls_mem[c].push_back(s);
    }
  }
  std::vector<int> sig_order;
  for (const auto& mem : cls_mem) sig_order.insert(sig_order.end(), mem.begin(), mem.end());
  th.nrows.assign(nm, 0);
  th.ncols.assign(nm, 0);
  th.base.assign(nm, 0);
  th.rowoff.assign(nm, std::vector<int64_t>(d, -1));
  th.coloff.assign(nm, std::vector<int64_t>(d, -1));
  for (int m = 0; m < nm; ++m) {
    for (int s1 : sig_order) {
      int s = A0.find(r.sub(th.mq[m], sigq[s1]));
      if (s < 0) continue;
      th.rowoff[m][s1] = th.nrows[m];
      th.nrows[m] += A0.sdim[s];
    }
    for (int s2 : sig_order) {
      int t = A2.find(r.add(th.mq[m], sigq[s2]));
      if (t < 0) continue;
      th.coloff[m][s2] = th.ncols[m];
      th.ncols[m] += A2.sdim[t];
    }
    th.base[m] = th.total;
    th.total += th.nrows[m] * th.ncols[m];
  }
  default_windows();
  bt.mark("theta space");
  // ---- allowed indices, ARPACK order (DMRG_routines.cpp:808-824) ----
  // ARPACK order = ascending s1 + d a0 + d chiL (s2 + d a2).  Every entry of
  // sector block m is allowed, so a column (s2, a2) holds exactly the rows of
  // block m = q(a2) - q(s2), in ascending s1 + d a0 order: the maps follow
  // from one row list per block and one descriptor per column.
  full_length = (int64_t)d * A0.size() * d * A2.size();
  const int64_t chiL = A0.size();
  map_secs.assign(nm, MapSec{0, 0, 0, 0});
  map_rowlin.clear();
  map_rowth.clear();
  for (int m = 0; m < nm; ++m) {
    map_secs[m].rowstart = (int64_t)map_rowlin.size();
    for (int64_t a0 = 0; a0 < chiL; ++a0)
      for (int s1 = 0; s1 < d; ++s1) {
        if (r.add(sigq[s1], A0.sq[A0.esec[a0]]) != th.mq[m]) continue;
        map_rowlin.push_back(s1 + (int64_t)d * a0);
        map_rowth.push_back(th.rowoff[m][s1] + A0.epos[a0]);
      }
    map_secs[m].nrows = (int64_t)map_rowlin.size() - map_secs[m].rowstart;
    map_secs[m].base = th.base[m];
    map_secs[m].ncols = th.ncols[m];
    if (map_secs[m].nrows != th.nrows[m]) return fail(CMPS_ERR_STATE, "internal: sector row count mismatch");
  }
  map_cols.clear();
  n_allowed = 0;
  for (int64_t a2 = 0; a2 < A2.size(); ++a2) {
    const QKey qa2 = A2.sq[A2.esec[a2]];
    for (int s2 = 0; s2 < d; ++s2) {
      const int im = th.find(r.sub(qa2, sigq[s2]));
      if (im < 0) continue;
      map_cols.push_back(MapCol{s2 + (int64_t)d * a2, th.coloff[im][s2] + A2.epos[a2], n_allowed, im});
      n_allowed += th.nrows[im];
    }
  }
  if (n_allowed != th.total) return fail(CMPS_ERR_STATE, "internal: allowed count differs from sector total");

  bt.mark("ARPACK maps");
  // ---- LeftPart blocks: key (b1, s1', s1, a0-sector s) ----
  lp_off.clear();
  lp_blocks.clear();
  lp_terms.clear();
  // (block key, term) pairs sorted by key, terms of one key in W order: the
  // blocks come out in key order with the terms as a per-key list would
  // hold them, without a tree insert per term
  struct KeyTerm {
    std::array<int, 4> key;
    AxpyTerm t;
  };
  auto by_key = [](const KeyTerm& a, const KeyTerm& b) { return a.key < b.key; };
  std::vector<KeyTerm> lpt;
  lpt.reserve(W.size() * (size_t)std::min(A0.nsec(), 8));
  for (const WEntry& w : W) {
    for (int s = 0; s < A0.nsec(); ++s) {
      int64_t lo = L.off[(size_t)w.bl * A0.nsec() + s];
      if (lo < 0) continue;
      QKey m = r.add(sigq[w.s], A0.sq[s]);
      if (th.find(m) < 0 || th.find(r.add(m, bq[w.br])) < 0) continue;
      lpt.push_back(KeyTerm{{w.br, w.sp, w.s, s}, AxpyTerm{lo, w.wr, w.wi}});
    }
  }
  std::stable_sort(lpt.begin(), lpt.end(), by_key);
  int64_t lp_total = 0;
  for (size_t i = 0, j = 0; i < lpt.size(); i = j) {
    const std::array<int, 4> key = lpt[i].key;
    for (j = i; j < lpt.size() && lpt[j].key == key; ++j) {
    }
    int s = key[3];
    // partner sector: q(s') = q(s) + q(b0) = q(s) + q(s1) + q(b1) - q(s1')
    QKey qsp = r.sub(r.add(r.add(A0.sq[s], sigq[key[2]]), bq[key[0]]), sigq[key[1]]);
    int sp = A0.find(qsp);
    if (sp < 0) continue;
    int64_t len = A0.sdim[sp] * A0.sdim[s];
    lp_off.emplace_hint(lp_off.end(), key, lp_total);
    lp_blocks.push_back(AxpyBlock{lp_total, len, (int32_t)lp_terms.size(), (int32_t)(lp_terms.size() + (j - i))});
    for (size_t q = i; q < j; ++q) lp_terms.push_back(lpt[q].t);
    lp_total += len;
  }
  // ---- RightPart blocks: key (b1, s2, s2', a2-sector t) ----
  rp_off.clear();
  rp_blocks.clear();
  rp_terms.clear();
  std::vector<KeyTerm> rpt;
  rpt.reserve(W.size() * (size_t)std::min(A2.nsec(), 8));
  for (const WEntry& w : W) {
    for (int t = 0; t < A2.nsec(); ++t) {
      int64_t ro = R.off[(size_t)w.br * A2.nsec() + t];
      if (ro < 0) continue;
      QKey m = r.sub(A2.sq[t], sigq[w.s]);
      if (th.find(m) < 0 || th.find(r.add(m, bq[w.bl])) < 0) continue;
      rpt.push_back(KeyTerm{{w.bl, w.s, w.sp, t}, AxpyTerm{ro, w.wr, w.wi}});
    }
  }
  std::stable_sort(rpt.begin(), rpt.end(), by_key);
  int64_t rp_total = 0;
  for (size_t i = 0, j = 0; i < rpt.size(); i = j) {
    const std::array<int, 4> key = rpt[i].key;
    for (j = i; j < rpt.size() && rpt[j].key == key; ++j) {
    }
    int t = key[3];
    // q(t') = q(t) + q(b2) = q(t) + q(s2') + q(b1) - q(s2)
    QKey qtp = r.sub(r.add(r.add(A2.sq[t], sigq[key[2]]), bq[key[0]]), sigq[key[1]]);
    int tp = A2.find(qtp);
    if (tp < 0) continue;
    int64_t len = A2.sdim[t] * A2.sdim[tp];
    rp_off.emplace_hint(rp_off.end(), key, rp_total);
    rp_blocks.push_back(AxpyBlock{rp_total, len, (int32_t)rp_terms.size(), (int32_t)(rp_terms.size() + (j - i))});
    for (size_t q = i; q < j; ++q) rp_terms.push_back(rpt[q].t);
    rp_total += len;
  }
  bt.mark("LP/RP block lists");
  CMPS_TRY(LP.alloc(lp_total));
  CMPS_TRY(RP.alloc(rp_total));
  CMPS_TRY(upload_vec(lp_blocks, &d_lp_blocks, ctx->stream));
  CMPS_TRY(upload_vec(lp_terms, &d_lp_terms, ctx->stream));
  CMPS_TRY(upload_vec(rp_blocks, &d_rp_blocks, ctx->stream));
  CMPS_TRY(upload_vec(rp_terms, &d_rp_terms, ctx->stream));

  bt.mark("LP/RP alloc+upload");
  owned.assign(nm, 1);
  CMPS_TRY(build_plans());
  for (const AxpyBlock& b : lp_blocks)
    for (int q = b.t0; q < b.t1; ++q)
      if (b.dst_off + b.len > lp_total || lp_terms[q].src_off + b.len > L.data.len)
        return fail(CMPS_ERR_STATE, "LeftPart block range outside its buffer");
  for (const AxpyBlock& b : rp_blocks)
    for (int q = b.t0; q < b.t1; ++q)
      if (b.dst_off + b.len > rp_total || rp_terms[q].src_off + b.len > R.data.len)
        return fail(CMPS_ERR_STATE, "RightPart block range outside its buffer");
  // pack map: every column and row index inside its sector block
  for (const MapCol& c : map_cols)
    if (c.m < 0 || c.m >= nm || c.colth < 0 || c.colth >= th.ncols[c.m])
      return fail(CMPS_ERR_STATE, "pack map column outside the sector blocks");
  for (int m = 0; m < nm; ++m)
    for (int64_t i = 0; i < map_secs[m].nrows; ++i) {
      const int64_t rt = map_rowth[map_secs[m].rowstart + i];
      if (rt < 0 || rt >= th.nrows[m]) return fail(CMPS_ERR_STATE, "pack map row outside the sector blocks");
    }
  bt.mark("folded plans");
  CMPS_TRY(build_pack(ctx->stream));
  cudaStream_t st = ctx->stream;
  CMPS_TRY(launch_block_axpy(d_lp_blocks, (int)lp_blocks.size(), d_lp_terms, L.data, LP, st));
  CMPS_TRY(launch_block_axpy(d_rp_blocks, (int)rp_blocks.size(), d_rp_terms, R.data, RP, st));

  bt.mark("pack + LP/RP formation");
  // ---- canonical four-stage flop count ----
  {
    double f = 0.0;
    std::set<int> usedbl, usedbr;
    for (const WEntry& w : W) { usedbl.insert(w.bl); usedbr.insert(w.br); }
    for (int m = 0; m < nm; ++m)
      for (int s1 = 0; s1 < d; ++s1) {
        if (th.rowoff[m][s1] < 0) continue;
        int s = A0.find(r.sub(th.mq[m], sigq[s1]));
        for (int b0 : usedbl) {
          int64_t lo = L.off[(size_t)b0 * A0.nsec() + s];
          if (lo < 0) continue;
          int sp = L.partner[(size_t)b0 * A0.nsec() + s];
          f += 8.0 * A0.sdim[sp] * (double)A0.sdim[s] * th.ncols[m];            // L . theta
        }
        for (const WEntry& w : W) {
          if (w.s != s1) continue;
          int64_t lo = L.off[(size_t)w.bl * A0.nsec() + s];
          if (lo < 0) continue;
          int sp = L.partner[(size_t)w.bl * A0.nsec() + s];
          f += 8.0 * A0.sdim[sp] * (double)th.ncols[m];                          // W1
        }
      }
    for (int m = 0; m < nm; ++m)
      for (int s2 = 0; s2 < d; ++s2) {
        if (th.coloff[m][s2] < 0) continue;
        int t = A2.find(r.add(th.mq[m], sigq[s2]));
        for (const WEntry& w : W) {
          if (w.s != s2) continue;
          int mp = th.find(r.add(th.mq[m], bq[w.bl]));
          if (mp < 0) continue;
          f += 8.0 * th.nrows[mp] * (double)A2.sdim[t];                         // W2
        }
        for (int b2 : usedbr) {
          int64_t ro = R.off[(size_t)b2 * A2.nsec() + t];
          if (ro < 0) continue;
          int tp = R.partner[(size_t)b2 * A2.nsec() + t];
          f += 8.0 * th.nrows[m] * (double)A2.sdim[t] * A2.sdim[tp];             // . R
        }
      }
    flops_canonical = f;
  }
  bt.mark("flop count");
  CMPS_TRY(x.alloc(th.total));
  CMPS_TRY(y.alloc(th.total));
  CMPS_CUDA(dmalloc(&d_io, sizeof(double) * 2 * std::max<int64_t>(1, n_allowed)));
  CMPS_TRY(ops.init(th.total));
  bt.mark("work vectors");
  CMPS_TRY(select_order());
  CMPS_CUDA(cudaStreamSynchronize(st));
  bt.mark("contraction order");
  return CMPS_OK;
}

// The FP64 matvec's contraction order: the one requested, or with
// CMPS_ORDER_AUTO the canonical order when it executes at most half the
// folded order's flops (it moves three intermediates through HBM where the
// folded order moves one, so a small flop advantage does not pay).
int Heff::select_order() {
  flops_folded = flops_executed;
  std::vector<uint8_t> cneed;
  CMPS_TRY(canonical_flops(*this, &flops_canon, &cneed));
  // the input sectors of either order (the windows must hold both)
  for (size_t m = 0; m < cneed.size() && m < in_need.size(); ++m) in_need[m] |= cneed[m];
  int want = order_req;
  if (want == CMPS_ORDER_AUTO) want = flops_canon <= 0.5 * flops_folded ? CMPS_ORDER_CANONICAL : CMPS_ORDER_FOLDED;
  // the canonical plans are rebuilt (or dropped), and the split-precision
  // operator, whose form follows the order, is prepared again
  release_split(this);
  if (want == CMPS_ORDER_CANONICAL) {
    CMPS_TRY(build_canonical(*this));
  } else {
    release_canonical(this);
  }
  order = want;
  if (is_split(precision)) CMPS_TRY(prepare_precision(this, precision));
  return CMPS_OK;
}

// The two grouped-GEMM plans of the matvec and the intermediate T, for the
// output sectors marked in `owned` (all of them unless the matvec is
// sharded): stage-2 tasks of owned output sectors only, and stage-1 tasks
// only for the blocks T^{b1}_m those read (m + q(b1) owned).
int Heff::build_plans() {
  const Rules& r = rules;
  const Bond& A0 = L.a;
  const Bond& A2 = R.a;
  const int nm = (int)th.mq.size();
  if ((int)owned.size() != nm) return fail(CMPS_ERR_STATE, "owned-sector mask size");
  stage1.release();
  stage2.release();
  T.release();
  if ((int)in_base.size() != nm || (int)out_base.size() != nm) return fail(CMPS_ERR_STATE, "window size");
  in_need.assign(nm, 0);
  // Dense (b, sigma', sigma, sector) -> block offset tables of lp_off /
  // rp_off for the plan loops below (several lookups per (b, m, sigma',
  // sigma)), when they stay small; the maps otherwise.
  const int64_t nlp = (int64_t)D * d * d * A0.nsec(), nrp = (int64_t)D * d * d * A2.nsec();
  constexpr int64_t kDenseMax = int64_t(1) << 24;
  std::vector<int64_t> lp_tab, rp_tab;
  if (nlp <= kDenseMax) {
    lp_tab.assign(nlp, -1);
    for (auto& kv2 : lp_off)
      lp_tab[(((int64_t)kv2.first[0] * d + kv2.first[1]) * d + kv2.first[2]) * A0.nsec() + kv2.first[3]] = kv2.second;
  }
  if (nrp <= kDenseMax) {
    rp_tab.assign(nrp, -1);
    for (auto& kv2 : rp_off)
      rp_tab[(((int64_t)kv2.first[0] * d + kv2.first[1]) * d + kv2.first[2]) * A2.nsec() + kv2.first[3]] = kv2.second;
  }
  auto lp_at = [&](int b, int sp, int sg, int sec) -> int64_t {
    if (!lp_tab.empty()) return lp_tab[(((int64_t)b * d + sp) * d + sg) * A0.nsec() + sec];
    auto it = lp_off.find({b, sp, sg, sec});
    return it == lp_off.end() ? -1 : it->second;
  };
  auto rp_at = [&](int b, int sg, int sp, int sec) -> int64_t {
    if (!rp_tab.empty()) return rp_tab[(((int64_t)b * d + sg) * d + sp) * A2.nsec() + sec];
    auto it = rp_off.find({b, sg, sp, sec});
    return it == rp_off.end() ? -1 : it->second;
  };
  // ---- stage 1: T^{b1}_m = LeftPart^{b1} . Theta_m ----
  std::set<int> b1s;
  for (auto& kv2 : lp_off) b1s.insert(kv2.first[0]);
  std::set<int> b1r;
  for (auto& kv2 : rp_off) b1r.insert(kv2.first[0]);
  t_base.assign((size_t)D * nm, -1);
  stage1 = GemmPlan();
  int64_t t_total = 0;
  flops_executed = 0.0;
  std::vector<double> fl(nm, 0.0);  // executed flops per output sector
  for (int b1 : b1s) {
    if (!b1r.count(b1)) continue;
    for (int m = 0; m < nm; ++m) {
      int mp = th.find(r.add(th.mq[m], bq[b1]));
      if (mp < 0 || !owned[mp]) continue;  // T^{b1}_m only feeds output sector mp
      std::vector<GemmTask> tasks;
      std::vector<GemmTerm> terms;
      int64_t ldc = th.ncols[m];
      for (int s1p = 0; s1p < d; ++s1p) {
        if (th.rowoff[mp][s1p] < 0) continue;
        int sp = A0.find(r.sub(th.mq[mp], sigq[s1p]));
        GemmTask task{};
        task.c_off = th.rowoff[mp][s1p] * ldc;  // relative to T block base, fixed below
        task.m = (int32_t)A0.sdim[sp];
        task.n = (int32_t)th.ncols[m];
        task.ldc = (int32_t)ldc;
        task.t0 = (int32_t)terms.size();
        for (int s1 = 0; s1 < d; ++s1) {
          if (th.rowoff[m][s1] < 0) continue;
          int s = A0.find(r.sub(th.mq[m], sigq[s1]));
          const int64_t lo = lp_at(b1, s1p, s1, s);
          if (lo < 0) continue;
          GemmTerm tm{};
          tm.a_off = lo;
          tm.lda = (int32_t)A0.sdim[s];
          tm.k = (int32_t)A0.sdim[s];
          if (in_base[m] < 0) return fail(CMPS_ERR_ARG, "input window lacks a sector the owned outputs read");
          tm.b_off = in_base[m] + th.rowoff[m][s1] * th.ncols[m];
          tm.ldb = (int32_t)th.ncols[m];
          terms.push_back(tm);
        }
        task.t1 = (int32_t)terms.size();
        tasks.push_back(task);
      }
      if (terms.empty()) continue;
      in_need[m] = 1;
      int64_t tb = t_total;
      t_base[(size_t)b1 * nm + m] = tb;
      t_total += th.nrows[mp] * th.ncols[m];
      int32_t term_base = (int32_t)stage1.terms.size();
      for (auto& tm : terms) {
        stage1.terms.push_back(tm);
      }
      for (auto& task : tasks) {
        task.c_off += tb;
        task.t0 += term_base;
        task.t1 += term_base;
        for (int q = task.t0; q < task.t1; ++q) {
          flops_executed += 8.0 * task.m * (double)task.n * stage1.terms[q].k;
          fl[mp] += 8.0 * task.m * (double)task.n * stage1.terms[q].k;
        }
        stage1.tasks.push_back(task);
      }
    }
  }
  t_len = t_total;  // T itself is allocated by the first folded FP64 matvec
  // ---- stage 2: Theta'_m' = sum_b1 T^{b1}_{m'-q(b1)} . RightPart^{b1} ----
  stage2 = GemmPlan();
  for (int mp = 0; mp < nm; ++mp) {
    if (!owned[mp]) continue;
    for (int s2p = 0; s2p < d; ++s2p) {
      if (th.coloff[mp][s2p] < 0) continue;
      int tp = A2.find(r.add(th.mq[mp], sigq[s2p]));
      GemmTask task{};
      if (out_base[mp] < 0) return fail(CMPS_ERR_ARG, "output window lacks an owned sector");
      task.c_off = out_base[mp] + th.coloff[mp][s2p];
      task.m = (int32_t)th.nrows[mp];
      task.n = (int32_t)A2.sdim[tp];
      task.ldc = (int32_t)th.ncols[mp];
      task.t0 = (int32_t)stage2.terms.size();
      for (int b1 = 0; b1 < D; ++b1) {
        int m = th.find(r.sub(th.mq[mp], bq[b1]));
        if (m < 0) continue;
        int64_t tb = t_base[(size_t)b1 * nm + m];
        if (tb < 0) continue;
        for (int s2 = 0; s2 < d; ++s2) {
          if (th.coloff[m][s2] < 0) continue;
          int t = A2.find(r.add(th.mq[m], sigq[s2]));
          const int64_t ro = rp_at(b1, s2, s2p, t);
          if (ro < 0) continue;
          GemmTerm tm{};
          tm.a_off = tb + th.coloff[m][s2];
          tm.lda = (int32_t)th.ncols[m];
          tm.k = (int32_t)A2.sdim[t];
          tm.b_off = ro;
          tm.ldb = (int32_t)A2.sdim[tp];
          stage2.terms.push_back(tm);
          flops_executed += 8.0 * task.m * (double)task.n * tm.k;
          fl[mp] += 8.0 * task.m * (double)task.n * tm.k;
        }
      }
      task.t1 = (int32_t)stage2.terms.size();
      stage2.tasks.push_back(task);
    }
  }
  CMPS_TRY(stage1.validate(false, false, LP.len, in_len, t_total, "stage 1"));
  CMPS_TRY(stage2.validate(false, false, t_total, RP.len, out_len, "stage 2"));
  if (all_owned()) sector_flops = fl;
  CMPS_TRY(stage1.upload(ctx->stream));
  CMPS_TRY(stage2.upload(ctx->stream));
  return CMPS_OK;
}

int Heff::autotune(TuneStats* stats) {
  cudaStream_t st = ctx->stream;
  if (is_split(precision) && !low_canonical) return CMPS_OK;
  CMPS_TRY(zero_wait(x.d, sizeof(double) * 2 * x.len, st));
  if (low_canonical && ctc) return CMPS_OK;  // tcgen05 stages: fixed tiles
  if (low_canonical) return autotune_canonical(*this, true, st, stats);
  if (order == CMPS_ORDER_CANONICAL) return autotune_canonical(*this, false, st, stats);
  CMPS_TRY(ensure_T());
  Planar in, out;
  in.d = x.d;
  in.len = in_len;
  out.d = y.d;
  out.len = out_len;
  int rc = autotune_plan(stage1, 1, [&] { return launch_zgemm_fp64(stage1, false, false, LP, in, T, st); }, st, stats);
  if (rc == CMPS_OK)
    rc = autotune_plan(stage2, 2, [&] { return launch_zgemm_fp64(stage2, false, false, T, RP, out, st); }, st, stats);
  in.d = out.d = nullptr;
  return rc;
}

void Heff::default_windows() {
  in_base = th.base;
  out_base = th.base;
  in_len = out_len = th.total;
  windowed = false;
}

int Heff::set_windows(const int64_t* ib, int64_t il, const int64_t* ob, int64_t ol) {
  const int nm = (int)th.mq.size();
  if (proj_np) return fail(CMPS_ERR_STATE, "windows: the projector term needs whole vectors");
  if (il < 0 || ol < 0) return fail(CMPS_ERR_ARG, "windows: negative length");
  for (int m = 0; m < nm; ++m) {
    const int64_t sz = th.nrows[m] * th.ncols[m];
    if (in_need[m] && (ib[m] < 0 || ib[m] + sz > il)) return fail(CMPS_ERR_ARG, "input window: a read sector is outside it");
    if (owned[m] && (ob[m] < 0 || ob[m] + sz > ol)) return fail(CMPS_ERR_ARG, "output window: an owned sector is outside it");
  }
  CMPS_CUDA(cudaStreamSynchronize(ctx->stream));
  in_base.assign(ib, ib + nm);
  out_base.assign(ob, ob + nm);
  for (int m = 0; m < nm; ++m) {
    if (!in_need[m]) in_base[m] = -1;
    if (!owned[m]) out_base[m] = -1;
  }
  in_len = il;
  out_len = ol;
  windowed = true;
  release_split(this);
  CMPS_TRY(build_plans());
  CMPS_TRY(select_order());
  if (is_split(precision)) CMPS_TRY(prepare_precision(this, precision));
  return CMPS_OK;
}

int Heff::set_owned(const uint8_t* mask) {
  const int nm = (int)th.mq.size();
  CMPS_CUDA(cudaStreamSynchronize(ctx->stream));
  default_windows();
  for (int m = 0; m < nm; ++m) owned[m] = mask[m] ? 1 : 0;
  release_split(this);
  CMPS_TRY(build_plans());
  CMPS_TRY(select_order());
  if (is_split(precision)) CMPS_TRY(prepare_precision(this, precision));
  return CMPS_OK;
}

bool Heff::all_owned() const {
  return std::all_of(owned.begin(), owned.end(), [](uint8_t o) { return o != 0; });
}

// The folded order's intermediate T: a canonical-order or split-precision
// handle never runs the folded FP64 stages, so T (about D x the wavefunction)
// is only allocated when they first run.
int Heff::ensure_T() {
  if (T.d && T.len == t_len) return CMPS_OK;
  return T.alloc(t_len);
}

// which = 1: the first half of the matvec (folded: T = LeftPart . in;
// canonical: stages L and W1), 2: the second half.
int Heff::apply_stage(int which, const Planar& in, Planar& out, cudaStream_t st) {
  if (is_split(precision)) return apply_split_stage(*this, which, in, out, st);
  if (order == CMPS_ORDER_CANONICAL) return apply_canonical(*this, which, in, out, st);
  CMPS_TRY(ensure_T());
  if (which == 1) return launch_zgemm_fp64(stage1, false, false, LP, in, T, st);
  return launch_zgemm_fp64(stage2, false, false, T, RP, out, st);
}

int Heff::apply_theta(const Planar& in, Planar& out, cudaStream_t st) {
  if (is_split(precision)) return apply_split(*this, in, out, st);
  CMPS_TRY(apply_stage(1, in, out, st));
  CMPS_TRY(apply_stage(2, in, out, st));
  return add_projectors(in, out, st);
}

int Heff::apply_fp64_stages(const Planar& in, Planar& out, cudaStream_t st) {
  if (order == CMPS_ORDER_CANONICAL) return apply_canonical(*this, 0, in, out, st);
  return apply_folded_fp64(in, out, st);
}

int Heff::apply_folded_fp64(const Planar& in, Planar& out, cudaStream_t st) {
  CMPS_TRY(ensure_T());
  CMPS_TRY(launch_zgemm_fp64(stage1, false, false, LP, in, T, st));
  CMPS_TRY(launch_zgemm_fp64(stage2, false, false, T, RP, out, st));
  return CMPS_OK;
}

int Heff::apply_theta_fp64(const Planar& in, Planar& out, cudaStream_t st) {
  CMPS_TRY(apply_fp64_stages(in, out, st));
  return add_projectors(in, out, st);
}

namespace {
// h[2p], h[2p+1] = -w_p * c_p (c_p = <phi_p, x>), for the subtracting multi-axpy
__global__ void k_proj_coef(const double* __restrict__ c, const double* __restrict__ w, int np,
                            double* __restrict__ h) {
  const int p = threadIdx.x;
  if (p < np) {
    h[2 * p] = -w[p] * c[2 * p];
    h[2 * p + 1] = -w[p] * c[2 * p + 1];
  }
}
}  // namespace

int Heff::set_projectors(int np, const double* host_arpack, const double* weights) {
  CMPS_CUDA(cudaStreamSynchronize(ctx->stream));
  proj.release();
  if (d_proj) dfree(d_proj);
  d_proj = nullptr;
  proj_np = 0;
  proj_w.clear();
  if (np == 0) return CMPS_OK;
  if (np < 0 || np > 64) return fail(CMPS_ERR_ARG, "projectors: between 0 and 64 of them");
  if (!host_arpack || !weights) return fail(CMPS_ERR_ARG, "projectors: null argument");
  if (windowed) return fail(CMPS_ERR_STATE, "projectors: the matvec has vector windows (sharded)");
  const int64_t n = th.total;
  CMPS_TRY(proj.alloc((int64_t)np * n));
  CMPS_CUDA(dmalloc(&d_proj, sizeof(double) * (3 * (size_t)np + 4)));
  cudaStream_t st = ctx->stream;
  std::vector<double> buf(2 * (size_t)n_allowed);
  for (int p = 0; p < np; ++p) {
    const double* src = host_arpack + 2 * (size_t)n_allowed * p;
    for (int64_t i = 0; i < n_allowed; ++i) {  // phi = conj(P)
      buf[2 * i] = src[2 * i];
      buf[2 * i + 1] = -src[2 * i + 1];
    }
    CMPS_TRY(copy_wait(d_io, buf.data(), sizeof(double) * 2 * n_allowed, cudaMemcpyHostToDevice, st));
    Planar v;
    v.d = proj.d + 2 * n * p;
    v.len = n;
    const int rc = pack(d_io, v, st);
    v.d = nullptr;
    CMPS_TRY(rc);
  }
  proj_w.assign(weights, weights + np);
  CMPS_TRY(copy_wait(d_proj, proj_w.data(), sizeof(double) * np, cudaMemcpyHostToDevice, st));
  CMPS_CUDA(cudaStreamSynchronize(st));
  proj_np = np;
  return CMPS_OK;
}

int Heff::set_projectors_device(int np, const double* d_phi_arpack, const double* weights) {
  CMPS_CUDA(cudaStreamSynchronize(ctx->stream));
  proj.release();
  if (d_proj) dfree(d_proj);
  d_proj = nullptr;
  proj_np = 0;
  proj_w.clear();
  if (np == 0) return CMPS_OK;
  if (np < 0 || np > 64) return fail(CMPS_ERR_ARG, "projectors: between 0 and 64 of them");
  if (!d_phi_arpack || !weights) return fail(CMPS_ERR_ARG, "projectors: null argument");
  const int64_t n = th.total;
  CMPS_TRY(proj.alloc((int64_t)np * n));
  CMPS_CUDA(dmalloc(&d_proj, sizeof(double) * (3 * (size_t)np + 4)));
  cudaStream_t st = ctx->stream;
  for (int p = 0; p < np; ++p) {
    Planar v;
    v.d = proj.d + 2 * n * p;
    v.len = n;
    const int rc = pack(d_phi_arpack + 2 * (size_t)n_allowed * p, v, st);
    v.d = nullptr;
    CMPS_TRY(rc);
  }
  proj_w.assign(weights, weights + np);
  CMPS_TRY(copy_wait(d_proj, proj_w.data(), sizeof(double) * np, cudaMemcpyHostToDevice, st));
  CMPS_CUDA(cudaStreamSynchronize(st));
  proj_np = np;
  return CMPS_OK;
}

int Heff::add_projectors(const Planar& in, Planar& out, cudaStream_t st) {
  if (!proj_np) return CMPS_OK;
  const int64_t n = th.total;
  // d_proj: weights [0, np), then c = <phi_p, x> (2 np) and |x|^2, then one
  // scratch norm; the coefficients are turned into -w_p c_p in place
  double* c = d_proj + proj_np;
  CMPS_TRY(ops.mdot_dev(proj.d, proj.d + n, 2 * n, proj_np, in.re(), in.im(), c, st));
  k_proj_coef<<<1, 64, 0, st>>>(c, d_proj, proj_np, c);
  CMPS_CUDA(cudaGetLastError());
  return ops.maxpy_norm_dev(proj.d, proj.d + n, 2 * n, proj_np, c, out.re(), out.im(), c + 2 * proj_np + 1, st);
}

int Heff::apply_device(const double* din, double* dout, cudaStream_t st) {
  if (!whole()) return fail(CMPS_ERR_STATE, "matvec is sharded: use the theta-layout entry point");
  CMPS_TRY(pack(din, x, st));
  if (is_split(precision)) {
    CMPS_TRY(apply_split_stage(*this, 1, x, y, st));
    CMPS_TRY(apply_split_stage(*this, 2, x, y, st));
    CMPS_TRY(add_projectors(x, y, st));
  } else {
    CMPS_TRY(apply_theta(x, y, st));
  }
  CMPS_TRY(unpack(y, dout, st));
  return CMPS_OK;
}

int Heff::apply_host(const double* in, double* out) {
  cudaStream_t st = ctx->stream;
  size_t bytes = sizeof(double) * 2 * n_allowed;
  CMPS_CUDA(cudaMemcpyAsync(d_io, in, bytes, cudaMemcpyHostToDevice, st));
  CMPS_TRY(apply_device(d_io, d_io, st));
  CMPS_CUDA(cudaMemcpyAsync(out, d_io, bytes, cudaMemcpyDeviceToHost, st));
  CMPS_CUDA(cudaStreamSynchronize(st));
  if (is_split(precision)) CMPS_TRY(split_error(*this));
  return CMPS_OK;
}

// ---------------------------------------------------------------------------
// Lowest eigenpair of the symmetric tridiagonal matrix with diagonal a[0..k)
// and off-diagonal b[0..k-1): the eigenvalue by Sturm-sequence bisection,
// the vector by two steps of inverse iteration with a row-pivoted
// tridiagonal LU.  O(k) per bisection step, so it runs after every Lanczos
// step.
static void tridiag_lowest(int k, const double* a, const double* b, double* lam, std::vector<double>& y) {
  y.assign(k, 0.0);
  if (k == 1) {
    *lam = a[0];
    y[0] = 1.0;
    return;
  }
  double lo = a[0], hi = a[0];
  for (int i = 0; i < k; ++i) {
    const double r = (i > 0 ? std::fabs(b[i - 1]) : 0.0) + (i + 1 < k ? std::fabs(b[i]) : 0.0);
    lo = std::min(lo, a[i] - r);
    hi = std::max(hi, a[i] + r);
  }
  const double eps = 2.220446049250313e-16;
  const double scale = std::max({std::fabs(lo), std::fabs(hi), 1e-300});
  const double pivmin = eps * scale;
  // number of eigenvalues below x (signs of the LDL^T pivots of T - x)
  auto below = [&](double x) {
    int c = 0;
    double d = 1.0;
    for (int i = 0; i < k; ++i) {
      double q = a[i] - x - (i > 0 ? b[i - 1] * b[i - 1] / d : 0.0);
      if (std::fabs(q) < pivmin) q = -pivmin;
      if (q < 0.0) ++c;
      d = q;
    }
    return c;
  };
  lo -= pivmin;
  hi += pivmin;
  for (int it = 0; it < 200 && hi - lo > 2.0 * eps * scale; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (below(mid) >= 1) hi = mid;
    else lo = mid;
  }
  *lam = 0.5 * (lo + hi);
  // inverse iteration: (T - lam) z = r
  std::vector<double> d(k), dl(k), du(k), du2(k), z(k, 1.0);
  std::vector<char> swapped(k, 0);
  for (int i = 0; i < k; ++i) d[i] = a[i] - *lam;
  for (int i = 0; i + 1 < k; ++i) dl[i] = du[i] = b[i];
  for (int i = 0; i + 1 < k; ++i) {
    du2[i] = 0.0;
    if (std::fabs(d[i]) >= std::fabs(dl[i])) {
      if (d[i] == 0.0) d[i] = pivmin;
      const double f = dl[i] / d[i];
      dl[i] = f;
      d[i + 1] -= f * du[i];
    } else {
      // exchange rows i and i+1
      const double f = d[i] / dl[i];
      d[i] = dl[i];
      dl[i] = f;
      const double t = du[i];
      du[i] = d[i + 1];
      d[i + 1] = t - f * d[i + 1];
      if (i + 2 < k) {
        du2[i] = du[i + 1];
        du[i + 1] = -f * du[i + 1];
      }
      swapped[i] = 1;
    }
  }
  if (d[k - 1] == 0.0) d[k - 1] = pivmin;
  for (int pass = 0; pass < 2; ++pass) {
    for (int i = 0; i + 1 < k; ++i) {
      if (!swapped[i]) {
        z[i + 1] -= dl[i] * z[i];
      } else {
        const double t = z[i] - dl[i] * z[i + 1];
        z[i] = z[i + 1];
        z[i + 1] = t;
      }
    }
    z[k - 1] /= d[k - 1];
    z[k - 2] = (z[k - 2] - du[k - 2] * z[k - 1]) / d[k - 2];
    for (int i = k - 3; i >= 0; --i) z[i] = (z[i] - du[i] * z[i + 1] - du2[i] * z[i + 2]) / d[i];
    double nz = 0.0;
    for (double v : z) nz += v * v;
    nz = std::sqrt(nz);
    for (double& v : z) v /= nz;
  }
  y = z;
}

// Restarted Lanczos with full re-orthogonalisation (the local three-term
// step, then one classical Gram-Schmidt pass against the whole basis),
// coefficients kept on the device and a convergence check after every step.
//
// FP64 operator: every step uses the FP64 matvec; the run ends when the Ritz
// residual estimate |beta_j y_j| falls below tol |lambda|.
//
// Split-TF32 operator (accurate to ~1e-5 relative): every restart cycle
// opens with an FP64 matvec of its start vector x, which gives the FP64
// Rayleigh quotient alpha_0 and the true residual beta_0 = |H x - alpha_0 x|;
// the run ends there once beta_0 <= tol |alpha_0|, with energy alpha_0.  The
// remaining steps of a cycle use the split operator and stop once the Ritz
// estimate has dropped by the cycle's factor eta_c below beta_0 (adapted
// from cycle to cycle, as described where it is declared).  A cycle therefore
// contracts the error of x by about max(eta, |dH| / gap) at the cost of one
// FP64 matvec, as in mixed-precision iterative refinement; if two cycles in a
// row fail to halve beta_0, the remaining cycles run in FP64.
int Heff::eigs(const double* guess, double tol, int max_restarts, int kdim, double* eval, double* evec,
               int* matvecs, bool start_in_x) {
  cudaStream_t st = ctx->stream;
  const int64_t n = th.total;
  if (n == 0) return fail(CMPS_ERR_STATE, "empty effective Hamiltonian");
  if (!whole()) return fail(CMPS_ERR_STATE, "matvec is sharded: the single-GPU eigensolver needs every sector");
  if (kdim < 2) kdim = 2;
  if (kdim > 96) kdim = 96;
  if ((int64_t)kdim > n) kdim = (int)n;
  if (kv_dim != kdim || kv.len != (int64_t)kdim * n) {
    CMPS_TRY(kv.alloc((int64_t)kdim * n));
    kv_dim = kdim;
  }
  if (!h_ab) CMPS_CUDA(cudaMallocHost(&h_ab, sizeof(double) * 4));
  const int64_t ldv = 2 * n;
  auto vre = [&](int j) { return kv.d + (int64_t)j * ldv; };
  auto view = [&](int j) {
    Planar p;
    p.d = vre(j);
    p.len = n;
    return p;
  };
  double* hA = ops.d_coef;        // 2 * 129
  double* hB = hA + 260;          // 2 * 129
  double* nrm = hA + 520;
  double* alpha_d = hA + 528;     // 128
  double* beta_d = hA + 656;      // 128
  double* scale_d = hA + 784;
  eig_stats = EigStats{};
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  struct EvGuard {
    cudaEvent_t* e;
    ~EvGuard() {
      for (int i = 0; i < 4; ++i)
        if (e[i]) cudaEventDestroy(e[i]);
    }
  } ev_guard{ev};
  for (auto& e : ev) CMPS_CUDA(cudaEventCreate(&e));
  CMPS_CUDA(cudaEventRecord(ev[2], st));
  // start vector into x
  if (guess) {
    CMPS_CUDA(cudaMemcpyAsync(d_io, guess, sizeof(double) * 2 * n_allowed, cudaMemcpyHostToDevice, st));
    CMPS_TRY(pack(d_io, x, st));
  }
  double nrm0 = 0.0;
  const bool have_start = guess || start_in_x;
  if (have_start) CMPS_TRY(ops.norm2(x.re(), x.im(), &nrm0, st));
  if (!have_start || !(nrm0 > 1e-300)) CMPS_TRY(ops.random(x.re(), x.im(), 0x5eed1234ULL, st));
  CMPS_TRY(ops.mdot_dev(nullptr, nullptr, 0, 0, x.re(), x.im(), nrm, st));
  CMPS_TRY(ops.scale_dev(x.re(), x.im(), nrm, true, x.re(), x.im(), st));

  const bool mixed = is_split(precision);
  if (mixed) CMPS_TRY(split_reset_error(*this, st));
  bool all_fp64 = !mixed;
  const int max_cycles = std::max(1, max_restarts) * (mixed ? 4 : 1);
  // Per-cycle contraction asked of the split steps.  A cycle's FP64 residual
  // shows what the previous cycle's split steps achieved: if they reached
  // their request, the next request is 30x stronger; if not, they met the
  // floor |dH|/gap of the split operator (or the Krylov cap), and the next
  // request is what they achieved.  No cycle asks for more than the
  // tolerance still needs (with a margin of 10).
  double eta = 1e-3;
  double eta_c = eta, prev_eta_c = eta;
  double prev_beta0 = HUGE_VAL;
  int stalls = 0, nmv = 0;
  double lam = 0.0;
  bool converged = false;
  std::vector<double> al, be, ycoef;
  for (int cycle = 0; cycle < max_cycles && !converged; ++cycle) {
    ++eig_stats.cycles;
    CMPS_CUDA(cudaMemcpyAsync(vre(0), x.d, sizeof(double) * 2 * n, cudaMemcpyDeviceToDevice, st));
    al.clear();
    be.clear();
    int k = 0;
    double beta0 = -1.0;
    bool split_used = false;
    for (int j = 0; j < kdim; ++j) {
      const bool fp64 = all_fp64 || j == 0;
      Planar vj = view(j);
      CMPS_CUDA(cudaEventRecord(ev[0], st));
      if (fp64) {
        CMPS_TRY(apply_theta_fp64(vj, y, st));
      } else {
        CMPS_TRY(apply_split_async(*this, vj, y, st));
        split_used = true;
      }
      CMPS_CUDA(cudaEventRecord(ev[1], st));
      ++nmv;
      // local three-term step (y -= beta_{j-1} v_{j-1}, alpha = <v_j, y>,
      // y -= alpha v_j), then one full classical Gram-Schmidt pass against
      // v_0..v_j that removes what rounding and the split operator's
      // non-Hermitian error leave behind
      const double* vp = j > 0 ? vre(j - 1) : nullptr;
      CMPS_TRY(ops.axpy_dot_dev(vp, vp ? vp + n : nullptr, beta_d + (j > 0 ? j - 1 : 0), vre(j), vre(j) + n, y.re(),
                                y.im(), hA, st));
      CMPS_TRY(ops.update_mdot_dev(hA, vre(j), vre(j) + n, kv.d, kv.d + n, ldv, j + 1, y.re(), y.im(), hB, st));
      CMPS_TRY(ops.maxpy_norm_dev(kv.d, kv.d + n, ldv, j + 1, hB, y.re(), y.im(), nrm, st));
      CMPS_TRY(ops.lanczos_coef(hA, hB + 2 * j, nrm, j, alpha_d, beta_d, scale_d, st));
      if (j + 1 < kdim) CMPS_TRY(ops.scale_dev(y.re(), y.im(), scale_d, false, vre(j + 1), vre(j + 1) + n, st));
      CMPS_CUDA(cudaMemcpyAsync(h_ab, alpha_d + j, sizeof(double), cudaMemcpyDeviceToHost, st));
      CMPS_CUDA(cudaMemcpyAsync(h_ab + 1, beta_d + j, sizeof(double), cudaMemcpyDeviceToHost, st));
      CMPS_CUDA(cudaStreamSynchronize(st));
      float mv_ms = 0.f;
      CMPS_CUDA(cudaEventElapsedTime(&mv_ms, ev[0], ev[1]));
      if (fp64) {
        ++eig_stats.mv_fp64;
        eig_stats.ms_fp64 += mv_ms;
      } else {
        ++eig_stats.mv_split;
        eig_stats.ms_split += mv_ms;
      }
      const double a = h_ab[0], b = h_ab[1];
      al.push_back(a);
      be.push_back(b);
      k = j + 1;
      const bool exhausted = !(b > 1e-14 * std::max(1.0, std::fabs(a)));
      tridiag_lowest(k, al.data(), be.data(), &lam, ycoef);
      const double resid = exhausted ? 0.0 : std::fabs(b * ycoef[k - 1]);
      if (all_fp64) {
        if (resid <= tol * std::max(1.0, std::fabs(lam))) {
          converged = true;
          break;
        }
        continue;
      }
      if (j == 0) {
        beta0 = b;
        if (exhausted || b <= tol * std::max(1.0, std::fabs(a))) {
          converged = true;  // x is the eigenvector; alpha_0 its FP64 energy
          lam = a;
          break;
        }
        if (prev_beta0 < HUGE_VAL) {
          const double got = b / prev_beta0;
          if (got > 0.5) {
            if (++stalls >= 2) all_fp64 = true;
          } else {
            stalls = 0;
          }
          eta = got <= 2.0 * prev_eta_c ? std::max(1e-10, prev_eta_c * 0.03) : std::min(0.1, got);
        }
        eta_c = std::min(0.5, std::max(eta, 0.1 * tol * std::max(1.0, std::fabs(a)) / b));
        prev_beta0 = b;
        prev_eta_c = eta_c;
      } else if (exhausted || resid <= eta_c * beta0) {
        break;
      }
    }
    if (split_used) CMPS_TRY(split_error(*this));
    if (converged && !all_fp64 && k == 1) break;
    // Ritz vector x = sum_j y_j v_j, normalised
    CMPS_TRY(ops.combine(kv.d, kv.d + n, ldv, k, ycoef.data(), x.re(), x.im(), st));
    CMPS_TRY(ops.mdot_dev(nullptr, nullptr, 0, 0, x.re(), x.im(), nrm, st));
    CMPS_TRY(ops.scale_dev(x.re(), x.im(), nrm, true, x.re(), x.im(), st));
  }
  CMPS_CUDA(cudaEventRecord(ev[3], st));
  // HED post-processing (DMRG_routines.cpp:870-889)
  double mx2 = 0.0;
  int64_t imx = 0;
  CMPS_TRY(ops.absmax(x.re(), x.im(), &mx2, &imx, st));
  double mr = 0.0, mi = 0.0;
  CMPS_CUDA(cudaMemcpyAsync(&mr, x.re() + imx, sizeof(double), cudaMemcpyDeviceToHost, st));
  CMPS_CUDA(cudaMemcpyAsync(&mi, x.im() + imx, sizeof(double), cudaMemcpyDeviceToHost, st));
  CMPS_CUDA(cudaStreamSynchronize(st));
  double mabs = std::sqrt(mx2);
  // phase = |max| / max = conj(max) / |max|
  double pr = mr / mabs, pi = -mi / mabs;
  CMPS_TRY(ops.phase_drop(x.re(), x.im(), pr, pi, 2.220446049250313e-16 * mabs, st));
  if (theta.len != n) CMPS_TRY(theta.alloc(n));
  CMPS_CUDA(cudaMemcpyAsync(theta.d, x.d, sizeof(double) * 2 * n, cudaMemcpyDeviceToDevice, st));
  have_theta = true;
  if (evec) {
    CMPS_TRY(unpack(theta, d_io, st));
    CMPS_CUDA(cudaMemcpyAsync(evec, d_io, sizeof(double) * 2 * n_allowed, cudaMemcpyDeviceToHost, st));
  }
  CMPS_CUDA(cudaStreamSynchronize(st));
  float total_ms = 0.f;
  CMPS_CUDA(cudaEventElapsedTime(&total_ms, ev[2], ev[3]));
  eig_stats.ms_total = total_ms;
  *eval = lam;
  if (matvecs) *matvecs = nmv;
  if (!converged) return fail(CMPS_ERR_SOLVER, "Lanczos did not reach the requested residual");
  return CMPS_OK;
}

}  // namespace cmps
