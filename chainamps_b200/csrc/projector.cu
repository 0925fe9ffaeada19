// Excited-state projectors built on the device from stored states: the
// ProjectorBlocks of the reference (DMRG_routines.cpp:446-581) and the
// projector tensors of its excited-state finite DMRG (fDMRG_routines.cpp:
// 68-244, ExcitedStateFiniteDMRG).
//
// A stored state p is kept as its site tensors T_k[s] (a_in x a_out, one
// matrix per physical state s), conjugated, the window's singular values
// folded into the left window tensor: U diag(lambda) and V^dagger.  Any exact
// representation of the state gives the same projector, so the reference's
// left / right / lambda files are not needed.  Against the current state
// (left tensors A_k, right tensors B_j of the running sweep) the overlaps are
//
//   PL_k = sum_s T_k[s]^dag PL_{k-1} A_k[s]      (stored bond x current bond)
//   PR_j = sum_s conj(T[s]) PR_{j-1} B_j[s]^T    (from the right end)
//
// (ProjectorBlocks::move_right_two_vertex / move_left_two_vertex, :540-581),
// and the projector tensor of the current window (makePTensor, :532-537) is
//
//   P[s1, a0, s2, a2] = sum PL[p, a0] conj(T1[s1])[p, r] conj(T2[s2])[r, q] PR[q, a2],
//
// on the window's allowed entries.  The matvec then adds sum_p w_p (P_p . x)
// conj(P_p) (TwoVertexMPOMPSMultiply, :947-973; Heff::add_projectors).
//
// Every contraction runs on dense bond matrices with cuBLAS ZGEMMs (the bond
// dimensions of a sweep are small next to the window's H_eff).  PL and PR are
// cached per bond position and per stored state, keyed by the serial number
// of the factorisation that produced each current tensor, so a sweep step
// extends them by one site.
#include <cublas_v2.h>
#include <cuComplex.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <memory>
#include <vector>

#include "heff.h"

namespace cmps {

namespace {

using cplx = cuDoubleComplex;
const cplx kOne = {1.0, 0.0}, kZero = {0.0, 0.0};

int grid_of(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 32)); }

// Entry (r, c) of a row-major planar block lands in matrix sig (from the row
// map, or from the column map when rsig is null) at (rdst[r], cdst[c]) of a
// stack of column-major matrices, scaled by cscale[c] and conjugated on
// request.
__global__ void k_scatter_site(const double* __restrict__ re, const double* __restrict__ im, int64_t nr, int64_t nc,
                               const int32_t* __restrict__ rsig, const int32_t* __restrict__ csig,
                               const int64_t* __restrict__ rdst, const int64_t* __restrict__ cdst,
                               const double* __restrict__ cscale, int conj, cplx* __restrict__ dst, int64_t ld,
                               int64_t stride) {
  const int64_t n = nr * nc;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e / nc, c = e % nc;
    const int64_t sig = rsig ? rsig[r] : csig[c];
    const double f = cscale ? cscale[c] : 1.0;
    dst[sig * stride + rdst[r] + ld * cdst[c]] = make_cuDoubleComplex(re[e] * f, (conj ? -im[e] : im[e]) * f);
  }
}

// phi[i] = conj(P[s1, a0, s2, a2]) at the full index of allowed entry i
// (row s1 + d a0 of d chi0 rows, column s2 + d a2), from P_all with rows
// s1 chi0 + a0 and columns s2 chi2 + a2; interleaved complex output.
__global__ void k_gather_projector(const cplx* __restrict__ P, const int64_t* __restrict__ full, int64_t n, int d,
                                   int64_t chi0, int64_t chi2, double* __restrict__ out) {
  const int64_t vrows = (int64_t)d * chi0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t f = full[i];
    const int64_t row = f % vrows, col = f / vrows;
    const int64_t s1 = row % d, a0 = row / d, s2 = col % d, a2 = col / d;
    const cplx v = P[(s1 * chi0 + a0) + vrows * (s2 * chi2 + a2)];
    out[2 * i] = v.x;
    out[2 * i + 1] = -v.y;
  }
}

struct Mat {
  cplx* p = nullptr;
  int64_t r = 0, c = 0;
};

// d column-major matrices (cin x cout), consecutive
struct Site {
  int d = 0;
  int64_t cin = 0, cout = 0;
  cplx* m = nullptr;
  cplx* at(int s) const { return m + (int64_t)s * cin * cout; }
};

void free_mat(Mat& x) {
  if (x.p) dfree(x.p);
  x = Mat();
}
void free_site(Site& x) {
  if (x.m) dfree(x.m);
  x = Site();
}

struct Blas {
  cublasHandle_t h;
  int st = CMPS_OK;
  void gemm(cublasOperation_t ta, cublasOperation_t tb, int64_t m, int64_t n, int64_t k, const cplx* A, int64_t lda,
            const cplx* B, int64_t ldb, cplx beta, cplx* C, int64_t ldc) {
    if (st != CMPS_OK || m == 0 || n == 0) return;
    if (cublasZgemm(h, ta, tb, (int)m, (int)n, (int)k, &kOne, A, (int)lda, B, (int)ldb, &beta, C, (int)ldc) !=
        CUBLAS_STATUS_SUCCESS)
      st = fail(CMPS_ERR_CUDA, "projectors: cublasZgemm failed");
  }
  void batched(cublasOperation_t ta, cublasOperation_t tb, int64_t m, int64_t n, int64_t k, const cplx* A,
               int64_t lda, int64_t sa, const cplx* B, int64_t ldb, int64_t sb, cplx* C, int64_t ldc, int64_t sc,
               int count) {
    if (st != CMPS_OK || m == 0 || n == 0 || count == 0) return;
    if (cublasZgemmStridedBatched(h, ta, tb, (int)m, (int)n, (int)k, &kOne, A, (int)lda, sa, B, (int)ldb, sb, &kZero,
                                  C, (int)ldc, sc, count) != CUBLAS_STATUS_SUCCESS)
      st = fail(CMPS_ERR_CUDA, "projectors: cublasZgemmStridedBatched failed");
  }
};

int alloc_zero(cplx** p, int64_t n, cudaStream_t st) {
  if (dmalloc(p, sizeof(cplx) * (size_t)std::max<int64_t>(n, 1)) != cudaSuccess)
    return fail(CMPS_ERR_NOMEM, "projectors: device allocation failed");
  return zero_wait(*p, sizeof(cplx) * (size_t)std::max<int64_t>(n, 1), st);
}

// Scatter launches with their small device maps, freed on destruction.
struct Maps {
  std::vector<void*> bufs;
  ~Maps() {
    for (void* p : bufs) dfree(p);
  }
  template <class T>
  int up(const std::vector<T>& h, T** d, cudaStream_t st) {
    if (dmalloc((void**)d, sizeof(T) * std::max<size_t>(h.size(), 1)) != cudaSuccess)
      return fail(CMPS_ERR_NOMEM, "projectors: map allocation failed");
    bufs.push_back(*d);
    if (h.empty()) return CMPS_OK;
    return copy_wait(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, st);
  }
};

// The left tensor U of a factorisation as a dense site: U[s1][a0, j] with j
// the new bond's element (global index); lam (by global index, may be empty)
// scales column j.
int site_from_u(const SvdResult& S, const std::vector<double>& lam, bool conj, cudaStream_t st, Site& out) {
  const ThetaSpace& th = S.th;
  out.d = S.d;
  out.cin = S.a0.size();
  out.cout = (int64_t)S.values.size();
  CMPS_TRY(alloc_zero(&out.m, (int64_t)out.d * out.cin * out.cout, st));
  Maps mp;
  for (int m = 0; m < (int)th.mq.size(); ++m) {
    const int64_t k = S.kept[m];
    if (!k) continue;
    const int64_t R = th.nrows[m];
    std::vector<int32_t> rsig(R, -1);
    std::vector<int64_t> rdst(R, -1), kcol(k);
    std::vector<double> ks(k, 1.0);
    for (int s1 = 0; s1 < S.d; ++s1) {
      if (th.rowoff[m][s1] < 0) continue;
      const int sa = S.a0.find(S.rules.sub(th.mq[m], S.sigq[s1]));
      if (sa < 0) return fail(CMPS_ERR_STATE, "projectors: left tensor row map");
      for (int64_t p = 0; p < S.a0.sdim[sa]; ++p) {
        rsig[th.rowoff[m][s1] + p] = s1;
        rdst[th.rowoff[m][s1] + p] = S.a0.selem[sa][p];
      }
    }
    for (int64_t j = 0; j < k; ++j) {
      kcol[j] = S.gidx[m][j];
      if (!lam.empty()) ks[j] = lam[S.gidx[m][j]];
      if (kcol[j] < 0 || kcol[j] >= out.cout) return fail(CMPS_ERR_STATE, "projectors: bond map");
    }
    for (int64_t r = 0; r < R; ++r)
      if (rsig[r] < 0 || rdst[r] < 0 || rdst[r] >= out.cin) return fail(CMPS_ERR_STATE, "projectors: left tensor row map");
    int32_t* d_rsig;
    int64_t *d_rdst, *d_kcol;
    double* d_ks;
    CMPS_TRY(mp.up(rsig, &d_rsig, st));
    CMPS_TRY(mp.up(rdst, &d_rdst, st));
    CMPS_TRY(mp.up(kcol, &d_kcol, st));
    CMPS_TRY(mp.up(ks, &d_ks, st));
    k_scatter_site<<<grid_of(R * k), 256, 0, st>>>(S.U.re() + S.uoff[m], S.U.im() + S.uoff[m], R, k, d_rsig, nullptr,
                                                   d_rdst, d_kcol, d_ks, conj ? 1 : 0, out.m, out.cin,
                                                   out.cin * out.cout);
    CMPS_CUDA(cudaGetLastError());
  }
  CMPS_CUDA(cudaStreamSynchronize(st));
  return CMPS_OK;
}

// The right tensor V^dagger as a dense site: Vd[s2][j, a2].
int site_from_vd(const SvdResult& S, bool conj, cudaStream_t st, Site& out) {
  const ThetaSpace& th = S.th;
  out.d = S.d;
  out.cin = (int64_t)S.values.size();
  out.cout = S.a2.size();
  CMPS_TRY(alloc_zero(&out.m, (int64_t)out.d * out.cin * out.cout, st));
  Maps mp;
  for (int m = 0; m < (int)th.mq.size(); ++m) {
    const int64_t k = S.kept[m];
    if (!k) continue;
    const int64_t C = th.ncols[m];
    std::vector<int32_t> csig(C, -1);
    std::vector<int64_t> cdst(C, -1), krow(k);
    for (int s2 = 0; s2 < S.d; ++s2) {
      if (th.coloff[m][s2] < 0) continue;
      const int t = S.a2.find(S.rules.add(th.mq[m], S.sigq[s2]));
      if (t < 0) return fail(CMPS_ERR_STATE, "projectors: right tensor column map");
      for (int64_t p = 0; p < S.a2.sdim[t]; ++p) {
        csig[th.coloff[m][s2] + p] = s2;
        cdst[th.coloff[m][s2] + p] = S.a2.selem[t][p];
      }
    }
    for (int64_t j = 0; j < k; ++j) {
      krow[j] = S.gidx[m][j];
      if (krow[j] < 0 || krow[j] >= out.cin) return fail(CMPS_ERR_STATE, "projectors: bond map");
    }
    for (int64_t q = 0; q < C; ++q)
      if (csig[q] < 0 || cdst[q] < 0 || cdst[q] >= out.cout)
        return fail(CMPS_ERR_STATE, "projectors: right tensor column map");
    int32_t* d_csig;
    int64_t *d_cdst, *d_krow;
    CMPS_TRY(mp.up(csig, &d_csig, st));
    CMPS_TRY(mp.up(cdst, &d_cdst, st));
    CMPS_TRY(mp.up(krow, &d_krow, st));
    k_scatter_site<<<grid_of(k * C), 256, 0, st>>>(S.Vd.re() + S.voff[m], S.Vd.im() + S.voff[m], k, C, nullptr, d_csig,
                                                   d_krow, d_cdst, nullptr, conj ? 1 : 0, out.m, out.cin,
                                                   out.cin * out.cout);
    CMPS_CUDA(cudaGetLastError());
  }
  CMPS_CUDA(cudaStreamSynchronize(st));
  return CMPS_OK;
}

int one_by_one(cudaStream_t st, Mat& x) {
  CMPS_TRY(alloc_zero(&x.p, 1, st));
  x.r = x.c = 1;
  return copy_wait(x.p, &kOne, sizeof(cplx), cudaMemcpyHostToDevice, st);
}

// PL' = sum_s Tc[s]^T PL A[s]  (Tc: the stored site, conjugated)
int left_overlap(Blas& b, cudaStream_t st, const Mat& PL, const Site& Tc, const Site& A, Mat& out) {
  if (PL.r != Tc.cin || PL.c != A.cin || Tc.d != A.d) return fail(CMPS_ERR_STATE, "projectors: left overlap shapes");
  cplx* W = nullptr;
  CMPS_TRY(alloc_zero(&W, (int64_t)A.d * PL.r * A.cout, st));
  out.r = Tc.cout;
  out.c = A.cout;
  int rc = alloc_zero(&out.p, out.r * out.c, st);
  if (rc == CMPS_OK) {
    b.batched(CUBLAS_OP_N, CUBLAS_OP_N, PL.r, A.cout, PL.c, PL.p, PL.r, 0, A.m, A.cin, A.cin * A.cout, W, PL.r,
              PL.r * A.cout, A.d);
    for (int s = 0; s < A.d; ++s)
      b.gemm(CUBLAS_OP_T, CUBLAS_OP_N, out.r, out.c, PL.r, Tc.at(s), Tc.cin, W + (int64_t)s * PL.r * A.cout, PL.r,
             s ? kOne : kZero, out.p, out.r);
    rc = b.st;
    if (rc == CMPS_OK && cudaStreamSynchronize(st) != cudaSuccess) rc = fail(CMPS_ERR_CUDA, "projectors: left overlap");
  }
  dfree(W);
  return rc;
}

// PR' = sum_s Tc[s] PR B[s]^T
int right_overlap(Blas& b, cudaStream_t st, const Mat& PR, const Site& Tc, const Site& B, Mat& out) {
  if (PR.r != Tc.cout || PR.c != B.cout || Tc.d != B.d) return fail(CMPS_ERR_STATE, "projectors: right overlap shapes");
  const int d = B.d;
  cplx* V = nullptr;  // rows s rp + i, ld d rp: the K-stack of PR B[s]^T
  CMPS_TRY(alloc_zero(&V, (int64_t)d * PR.r * B.cin, st));
  out.r = Tc.cin;
  out.c = B.cin;
  int rc = alloc_zero(&out.p, out.r * out.c, st);
  if (rc == CMPS_OK) {
    b.batched(CUBLAS_OP_N, CUBLAS_OP_T, PR.r, B.cin, PR.c, PR.p, PR.r, 0, B.m, B.cin, B.cin * B.cout, V,
              (int64_t)d * PR.r, PR.r, d);
    b.gemm(CUBLAS_OP_N, CUBLAS_OP_N, out.r, out.c, (int64_t)d * PR.r, Tc.m, Tc.cin, V, (int64_t)d * PR.r, kZero, out.p,
           out.r);
    rc = b.st;
    if (rc == CMPS_OK && cudaStreamSynchronize(st) != cudaSuccess) rc = fail(CMPS_ERR_CUDA, "projectors: right overlap");
  }
  dfree(V);
  return rc;
}

}  // namespace

struct ProjectedState {
  double weight = 0.0;
  std::vector<Site> site;  // conj(T_k), k = 0 .. length - 1
  // overlap caches: pl[k] after k left sites, made with the current left
  // tensors of serials pl_src[1..k]; pr[j] likewise from the right end
  std::vector<Mat> pl, pr;
  std::vector<uint64_t> pl_src, pr_src;
  ~ProjectedState() {
    for (auto& s : site) free_site(s);
    for (auto& m : pl) free_mat(m);
    for (auto& m : pr) free_mat(m);
  }
};

void projected_state_destroy(ProjectedState* p) { delete p; }

int projected_state_create(cmps_context* ctx, const std::map<int64_t, std::shared_ptr<SvdResult>>& lsvd,
                           const std::map<int64_t, std::shared_ptr<SvdResult>>& rsvd, const SvdResult& window,
                           const std::vector<double>& lambda, int64_t nleft, int64_t length, double weight,
                           ProjectedState** out) {
  *out = nullptr;
  cudaStream_t st = ctx->stream;
  const int64_t nright = length - nleft - 2;
  if (nleft < 0 || nright < 0) return fail(CMPS_ERR_STATE, "projected state: no two-vertex window");
  std::unique_ptr<ProjectedState> p(new ProjectedState());
  p->weight = weight;
  p->site.resize((size_t)length);
  for (int64_t k = 1; k <= nleft; ++k) {
    auto it = lsvd.find(k);
    if (it == lsvd.end() || !it->second) return fail(CMPS_ERR_STATE, "projected state: a left tensor is missing");
    CMPS_TRY(site_from_u(*it->second, {}, true, st, p->site[k - 1]));
  }
  CMPS_TRY(site_from_u(window, lambda, true, st, p->site[nleft]));
  CMPS_TRY(site_from_vd(window, true, st, p->site[nleft + 1]));
  for (int64_t k = nleft + 2; k < length; ++k) {
    auto it = rsvd.find(length - k);
    if (it == rsvd.end() || !it->second) return fail(CMPS_ERR_STATE, "projected state: a right tensor is missing");
    CMPS_TRY(site_from_vd(*it->second, true, st, p->site[k]));
  }
  for (int64_t k = 0; k + 1 < length; ++k)
    if (p->site[k].cout != p->site[k + 1].cin) return fail(CMPS_ERR_STATE, "projected state: bonds do not chain");
  p->pl.resize(1);
  p->pr.resize(1);
  p->pl_src.assign(1, 0);
  p->pr_src.assign(1, 0);
  CMPS_TRY(one_by_one(st, p->pl[0]));
  CMPS_TRY(one_by_one(st, p->pr[0]));
  *out = p.release();
  return CMPS_OK;
}

// The projector tensors of every stored state for the window of H (the
// current state's left tensors lsvd[1..nleft], right tensors
// rsvd[1..nright]), installed as H's projectors.
int install_projectors(cmps_context* ctx, std::vector<ProjectedState*>& states,
                       const std::map<int64_t, std::shared_ptr<SvdResult>>& lsvd,
                       const std::map<int64_t, std::shared_ptr<SvdResult>>& rsvd, int64_t nleft, int64_t length,
                       Heff& H) {
  if (states.empty()) return H.set_projectors_device(0, nullptr, nullptr);
  cudaStream_t st = ctx->stream;
  void* bv = nullptr;
  CMPS_TRY(context_blas(ctx, &bv));
  Blas b{(cublasHandle_t)bv};
  const int64_t nright = length - nleft - 2;
  const int d = H.d;
  const int64_t chi0 = H.L.a.size(), chi2 = H.R.a.size(), n = H.n_allowed;
  if ((int64_t)d * chi0 * d * chi2 != H.full_length) return fail(CMPS_ERR_STATE, "projectors: window shape");
  // the current tensors' serial numbers, checked against the caches
  std::vector<uint64_t> lser(nleft + 1, 0), rser(nright + 1, 0);
  for (int64_t k = 1; k <= nleft; ++k) {
    auto it = lsvd.find(k);
    if (it == lsvd.end() || !it->second) return fail(CMPS_ERR_STATE, "projectors: a current left tensor is missing");
    lser[k] = it->second->serial;
  }
  for (int64_t j = 1; j <= nright; ++j) {
    auto it = rsvd.find(j);
    if (it == rsvd.end() || !it->second) return fail(CMPS_ERR_STATE, "projectors: a current right tensor is missing");
    rser[j] = it->second->serial;
  }
  int64_t* d_full = nullptr;
  double* d_phi = nullptr;
  if (dmalloc(&d_full, sizeof(int64_t) * (size_t)std::max<int64_t>(n, 1)) != cudaSuccess)
    return fail(CMPS_ERR_NOMEM, "projectors: index map allocation failed");
  if (dmalloc(&d_phi, sizeof(double) * 2 * (size_t)std::max<int64_t>(n, 1) * states.size()) != cudaSuccess) {
    dfree(d_full);
    return fail(CMPS_ERR_NOMEM, "projectors: tensor allocation failed");
  }
  int rc = H.arpack_map(1, d_full, st);
  std::vector<double> weights;
  for (size_t ip = 0; ip < states.size() && rc == CMPS_OK; ++ip) {
    ProjectedState& P = *states[ip];
    if ((int64_t)P.site.size() != length) {
      rc = fail(CMPS_ERR_STATE, "projectors: a stored state has another length");
      break;
    }
    weights.push_back(P.weight);
    // ---- PL up to nleft ----
    int64_t j = 0;
    while (j < nleft && j + 1 < (int64_t)P.pl.size() && P.pl_src[j + 1] == lser[j + 1]) ++j;
    for (int64_t k = (int64_t)P.pl.size() - 1; k > j; --k) free_mat(P.pl[k]);
    P.pl.resize(j + 1);
    P.pl_src.resize(j + 1);
    for (int64_t k = j + 1; k <= nleft && rc == CMPS_OK; ++k) {
      Site A;
      rc = site_from_u(*lsvd.at(k), {}, false, st, A);
      Mat nx;
      if (rc == CMPS_OK) rc = left_overlap(b, st, P.pl[k - 1], P.site[k - 1], A, nx);
      free_site(A);
      if (rc != CMPS_OK) {
        free_mat(nx);
        break;
      }
      P.pl.push_back(nx);
      P.pl_src.push_back(lser[k]);
    }
    // ---- PR up to nright ----
    j = 0;
    while (rc == CMPS_OK && j < nright && j + 1 < (int64_t)P.pr.size() && P.pr_src[j + 1] == rser[j + 1]) ++j;
    if (rc == CMPS_OK) {
      for (int64_t k = (int64_t)P.pr.size() - 1; k > j; --k) free_mat(P.pr[k]);
      P.pr.resize(j + 1);
      P.pr_src.resize(j + 1);
    }
    for (int64_t k = j + 1; k <= nright && rc == CMPS_OK; ++k) {
      Site B;
      rc = site_from_vd(*rsvd.at(k), false, st, B);
      Mat nx;
      if (rc == CMPS_OK) rc = right_overlap(b, st, P.pr[k - 1], P.site[length - k], B, nx);
      free_site(B);
      if (rc != CMPS_OK) {
        free_mat(nx);
        break;
      }
      P.pr.push_back(nx);
      P.pr_src.push_back(rser[k]);
    }
    if (rc != CMPS_OK) break;
    // ---- P on the window ----
    const Mat& PL = P.pl[nleft];
    const Mat& PR = P.pr[nright];
    const Site& T1 = P.site[nleft];
    const Site& T2 = P.site[nleft + 1];
    if (PL.c != chi0 || PR.c != chi2 || PL.r != T1.cin || PR.r != T2.cout || T1.d != d || T2.d != d) {
      rc = fail(CMPS_ERR_STATE, "projectors: overlap shapes do not match the window");
      break;
    }
    const int64_t chr = T1.cout;
    cplx *M1 = nullptr, *M2 = nullptr, *Pall = nullptr;
    rc = alloc_zero(&M1, (int64_t)d * chi0 * chr, st);
    if (rc == CMPS_OK) rc = alloc_zero(&M2, chr * (int64_t)d * chi2, st);
    if (rc == CMPS_OK) rc = alloc_zero(&Pall, (int64_t)d * chi0 * d * chi2, st);
    if (rc == CMPS_OK) {
      // M1[s1] = PL^T T1c[s1], rows s1 chi0 + a0 of a (d chi0) x chr matrix
      b.batched(CUBLAS_OP_T, CUBLAS_OP_N, chi0, chr, PL.r, PL.p, PL.r, 0, T1.m, T1.cin, T1.cin * T1.cout, M1,
                (int64_t)d * chi0, chi0, d);
      // M2[s2] = T2c[s2] PR, columns s2 chi2 + a2 of a chr x (d chi2) matrix
      b.batched(CUBLAS_OP_N, CUBLAS_OP_N, chr, chi2, PR.r, T2.m, T2.cin, T2.cin * T2.cout, PR.p, PR.r, 0, M2, chr,
                chr * chi2, d);
      b.gemm(CUBLAS_OP_N, CUBLAS_OP_N, (int64_t)d * chi0, (int64_t)d * chi2, chr, M1, (int64_t)d * chi0, M2, chr,
             kZero, Pall, (int64_t)d * chi0);
      rc = b.st;
    }
    if (rc == CMPS_OK) {
      k_gather_projector<<<grid_of(n), 256, 0, st>>>(Pall, d_full, n, d, chi0, chi2, d_phi + 2 * (size_t)n * ip);
      if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
        rc = fail(CMPS_ERR_CUDA, "projectors: gather failed");
    }
    if (M1) dfree(M1);
    if (M2) dfree(M2);
    if (Pall) dfree(Pall);
  }
  if (rc == CMPS_OK) rc = H.set_projectors_device((int)states.size(), d_phi, weights.data());
  dfree(d_full);
  dfree(d_phi);
  return rc;
}

}  // namespace cmps
