// Device-resident iDMRG growth (SuperBlock::grow_two_vertex,
// DMRG_routines.cpp:346-374): every step builds the new environments from the
// previous step's H_eff and SVD on the device (MakeLeftBlock / MakeRightBlock,
// :594-611), forms the new H_eff, predicts its start vector on the device
// (MakePrediction, :693-707), solves for the ground state and truncates.
// Nothing but scalars and singular values crosses to the host.
//
// Prediction: with U, s, V^dagger of the last step and lambda_prev of the one
// before, the guess for the next two-vertex wavefunction is
//   G(s1''=s2, k, s2''=s1, new) = s_k s_new sum_j V^dagger[k,(s2,j)] U[(s1,j),new] / lambda_prev[j]
// (the contraction of ALambdaR, the inverse previous lambda and LambdaLB in
// MakePrediction), computed as one grouped FP64 GEMM into the new theta blocks.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>

#include "heff.h"

namespace cmps {

namespace {

// out[r, c] = in[r, c] * rs[r] * cs[c] over one row-major block
__global__ void k_scale_block(const double* __restrict__ ir, const double* __restrict__ ii, int64_t rows, int64_t cols,
                              const double* __restrict__ rs, const double* __restrict__ cs, double* __restrict__ orr,
                              double* __restrict__ oi) {
  const int64_t n = rows * cols;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e / cols, c = e % cols;
    const double f = (rs ? rs[r] : 1.0) * (cs ? cs[c] : 1.0);
    orr[e] = ir[e] * f;
    oi[e] = ii[e] * f;
  }
}

int grid_n(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16)); }

double entropy_of(const std::vector<double>& v) {
  double s = 0.0;
  for (double x : v)
    if (x != 0.0) s -= x * x * std::log(x * x);
  return s;
}

}  // namespace

struct Dmrg {
  cmps_context* ctx = nullptr;
  int device = 0;
  Rules rules;
  int precision = CMPS_FP64;
  // deep copy of the MPO descriptor
  std::vector<uint8_t> w_in, w_ph;
  std::vector<int64_t> w_sz, w_cp, w_ri;
  std::vector<int16_t> w_ch;
  std::vector<double> w_val;
  cmps_mpx_desc W{};
  QKey target{};
  int D = 0;
  std::vector<QKey> bq;
  int64_t size = 0;
  std::unique_ptr<Heff> heff;
  std::shared_ptr<SvdResult> svd;  // factors of the current window (shared with lsvd / rsvd)
  static std::shared_ptr<SvdResult> new_svd() {
    static std::atomic<uint64_t> serials{0};
    auto p = std::shared_ptr<SvdResult>(new SvdResult(), [](SvdResult* s) {
      s->U.release();
      s->Vd.release();
      delete s;
    });
    p->serial = ++serials;
    return p;
  }
  std::vector<double> lambda, prev_lambda;
  double tol = 1e-10;
  int restarts = 50, kdim = 24;
  int last_matvecs = 0;
  double last_ms[4] = {0, 0, 0, 0};  // env update + H_eff build + prediction, eigensolve, svd, total
  // coupling gradient: dW and the derivative environments of the current
  // window carried along (no device data: zero, as for the dummy blocks);
  // with kept blocks, the derivative blocks of every length beside them
  bool grad_on = false;
  std::vector<WEntry> dW;
  Env dL, dR;
  bool have_dlr = false;
  std::map<int64_t, Env> dlblocks, drblocks;
  const Env* dl_ptr() const { return dL.data.d ? &dL : nullptr; }
  const Env* dr_ptr() const { return dR.data.d ? &dR : nullptr; }
  // the current window's derivative environments from the kept ones
  int load_derivatives(int64_t nl, int64_t nr, cudaStream_t st) {
    dL.data.release();
    dR.data.release();
    dL = Env();
    dR = Env();
    auto il = dlblocks.find(nl);
    auto ir = drblocks.find(nr);
    if (il != dlblocks.end()) CMPS_TRY(copy_env(il->second, dL, st));
    if (ir != drblocks.end()) CMPS_TRY(copy_env(ir->second, dR, st));
    have_dlr = dL.data.d || dR.data.d;
    return CMPS_OK;
  }
  // the derivative of MakeLeftBlock (right = false) or MakeRightBlock with
  // this window's factors, stored beside the block of length k
  int store_derivative(bool right, int64_t k, cudaStream_t st) {
    Env nl, nr;
    int rc = derivative_envs(*heff, *svd, dW, dl_ptr(), dr_ptr(), nl, nr);
    if (rc == CMPS_OK) rc = store(right ? drblocks : dlblocks, k, right ? nr : nl, st);
    nl.data.release();
    nr.data.release();
    return rc;
  }
  double last_grad = std::nan("");
  static constexpr int kProfile = 21;
  double last_profile[kProfile] = {0};  // cmps_dmrg_profile layout

  // excited states: the states projected out of every solve (next_state,
  // fDMRG_routines.hpp:39-44), with their weights
  std::vector<ProjectedState*> pstates;
  ~Dmrg() {
    for (ProjectedState* p : pstates) projected_state_destroy(p);
    dL.data.release();
    dR.data.release();
    for (auto& kv : lblocks) kv.second.data.release();
    for (auto& kv : rblocks) kv.second.data.release();
    for (auto& kv : dlblocks) kv.second.data.release();
    for (auto& kv : drblocks) kv.second.data.release();
  }
  // finite sweeps: the blocks of every length, kept when keep_blocks is set
  // before growth; key = number of vertices the block covers
  bool keep_blocks = false;
  bool want_fidelity = true;  // CheckConvergence on growth steps
  int order_req = CMPS_ORDER_AUTO;  // contraction order of each step's H_eff
  bool autotune = false;            // measured tile shapes for each step's grouped GEMM plans
  TuneStats tune;                   // accumulated over the run
  std::map<int64_t, Env> lblocks, rblocks;
  // the factors each kept block was built with: lsvd[k]'s U made lblocks[k]
  // (the left MPS tensor of vertex k), rsvd[k]'s V^dagger made rblocks[k]
  // (the right MPS tensor of the k-th vertex from the right end)
  std::map<int64_t, std::shared_ptr<SvdResult>> lsvd, rsvd;
  int64_t nleft = 0;  // vertices left of the two-vertex window

  int dummy_blocks(Env& L, Env& R);
  int predict(Heff& next, bool* ok);
  int finite_predict(Heff& next, int dir, bool* ok);
  // dir 0: iDMRG growth step (grow_two_vertex); +1 / -1: finite sweep step
  // to the right / left (move_{right,left}_two_vertex); 2: a new solve of the
  // current window with its environments (ExcitedStateFiniteDMRG::init,
  // fDMRG_routines.cpp:68-91)
  int step(int dir, int64_t chi, double trunc, double* out);
  int project_state(double weight) {
    if (!keep_blocks || !svd || size < 2) return fail(CMPS_ERR_STATE, "projected state: run a finite chain first");
    ProjectedState* p = nullptr;
    CMPS_TRY(projected_state_create(ctx, lsvd, rsvd, *svd, lambda, nleft, size, weight, &p));
    pstates.push_back(p);
    return CMPS_OK;
  }
  int grow(int64_t chi, double trunc, double* out) { return step(0, chi, trunc, out); }
  static int store(std::map<int64_t, Env>& m, int64_t k, const Env& e, cudaStream_t st) {
    auto it = m.find(k);
    if (it != m.end()) it->second.data.release();
    Env c;
    CMPS_TRY(copy_env(e, c, st));
    m[k] = c;
    return CMPS_OK;
  }
};

int Dmrg::dummy_blocks(Env& L, Env& R) {
  // MakeDummyLeftBlock / MakeDummyRightBlock (DMRG_routines.cpp:613-653)
  const int nq = rules.nq;
  auto build = [&](bool right, Env& e) -> int {
    std::vector<uint8_t> in(6), ph(6, 0);
    std::vector<int64_t> sz(6, 1);
    std::vector<int16_t> ch;
    int ib = right ? 2 : 3;
    sz[ib] = D;
    if (!right) in = {0, 1, 1, 0, 1, 0};
    else in = {0, 1, 1, 0, 1, 0};
    for (int i = 0; i < 6; ++i) {
      for (int64_t k = 0; k < sz[i]; ++k)
        for (int c = 0; c < nq; ++c) {
          int16_t v = 0;
          if (i == ib) v = bq[k][c];
          else if (right && (i == 0 || i == 4)) v = target[c];
          ch.push_back(v);
        }
    }
    std::vector<int64_t> cp = {0, 1}, ri = {right ? 0 : (int64_t)(D - 1)};
    std::vector<double> val = {1.0, 0.0};
    cmps_mpx_desc d{6, right ? 3 : 4, in.data(), ph.data(), sz.data(), ch.data(), (int64_t)D, 1,
                    cp.data(), ri.data(), val.data()};
    return build_env_from_desc(rules, &d, right, e, D, bq, ctx->stream);
  };
  CMPS_TRY(build(false, L));
  CMPS_TRY(build(true, R));
  return CMPS_OK;
}

// Fill next.x with the prediction; *ok = false when it does not apply.
int Dmrg::predict(Heff& next, bool* ok) {
  *ok = false;
  if (!svd || prev_lambda.empty()) return CMPS_OK;
  const SvdResult& S = *svd;
  if (S.a0.element_charges() != S.a2.element_charges()) return CMPS_OK;  // pairing by position needs equal bonds
  if ((int64_t)prev_lambda.size() != S.a0.size()) return CMPS_OK;
  cudaStream_t st = ctx->stream;
  const ThetaSpace& to = S.th;       // previous theta space
  const ThetaSpace& tn = next.th;    // next theta space
  const int nmo = (int)to.mq.size();
  const int d = next.d;
  // scaled factors: Vs = diag(s) Vd ; Us = diag(1/lambda_prev) U diag(s)
  Planar Us, Vs;
  CMPS_TRY(Us.alloc(std::max<int64_t>(1, S.U.len)));
  CMPS_TRY(Vs.alloc(std::max<int64_t>(1, S.Vd.len)));
  std::vector<double> rs, cs;
  double* d_scale = nullptr;
  int status = CMPS_OK;
  for (int m = 0; m < nmo && status == CMPS_OK; ++m) {
    const int64_t k = S.kept[m];
    if (!k) continue;
    std::vector<double> colsc(k), urow(to.nrows[m], 0.0);
    for (int64_t j = 0; j < k; ++j) colsc[j] = lambda[S.gidx[m][j]];
    for (int s1 = 0; s1 < d; ++s1) {
      if (to.rowoff[m][s1] < 0) continue;
      int sa = S.a0.find(S.rules.sub(to.mq[m], S.sigq[s1]));
      for (int64_t p = 0; p < S.a0.sdim[sa]; ++p) {
        const double lp = prev_lambda[S.a0.selem[sa][p]];
        urow[to.rowoff[m][s1] + p] = lp != 0.0 ? 1.0 / lp : 0.0;
      }
    }
    const size_t nb = urow.size() + 2 * colsc.size();
    std::vector<double> hostbuf;
    hostbuf.insert(hostbuf.end(), urow.begin(), urow.end());
    hostbuf.insert(hostbuf.end(), colsc.begin(), colsc.end());
    hostbuf.insert(hostbuf.end(), colsc.begin(), colsc.end());
    if (dmalloc(&d_scale, sizeof(double) * nb) != cudaSuccess) {
      status = fail(CMPS_ERR_NOMEM, "prediction scale allocation failed");
      break;
    }
    if ((status = copy_wait(d_scale, hostbuf.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, st)) != CMPS_OK)
      break;
    const double* d_urow = d_scale;
    const double* d_ucol = d_scale + urow.size();
    const double* d_vrow = d_ucol + k;
    k_scale_block<<<grid_n(to.nrows[m] * k), 256, 0, st>>>(S.U.re() + S.uoff[m], S.U.im() + S.uoff[m], to.nrows[m],
                                                          k, d_urow, d_ucol, Us.re() + S.uoff[m],
                                                          Us.im() + S.uoff[m]);
    k_scale_block<<<grid_n(k * to.ncols[m]), 256, 0, st>>>(S.Vd.re() + S.voff[m], S.Vd.im() + S.voff[m], k,
                                                          to.ncols[m], d_vrow, nullptr, Vs.re() + S.voff[m],
                                                          Vs.im() + S.voff[m]);
    cudaStreamSynchronize(st);
    dfree(d_scale);
    d_scale = nullptr;
  }
  // grouped GEMM plan into the next theta blocks
  GemmPlan p;
  if (status == CMPS_OK) {
    for (int mn = 0; mn < (int)tn.mq.size(); ++mn)
      for (int a = 0; a < d; ++a) {            // sigma1'' = old sigma2
        if (tn.rowoff[mn][a] < 0) continue;
        const int mk = to.find(next.rules.sub(tn.mq[mn], next.sigq[a]));
        if (mk < 0 || !S.kept[mk] || to.coloff[mk][a] < 0) continue;
        for (int b = 0; b < d; ++b) {          // sigma2'' = old sigma1
          if (tn.coloff[mn][b] < 0) continue;
          const int mw = to.find(next.rules.add(tn.mq[mn], next.sigq[b]));
          if (mw < 0 || !S.kept[mw] || to.rowoff[mw][b] < 0) continue;
          const int t = S.a2.find(S.rules.add(to.mq[mk], S.sigq[a]));
          const int s = S.a0.find(S.rules.sub(to.mq[mw], S.sigq[b]));
          if (t < 0 || s < 0 || S.a2.sdim[t] != S.a0.sdim[s]) continue;
          // the next theta's row chunk must be exactly the kept states of block mk (and columns of mw)
          const int sr = next.L.a.find(to.mq[mk]);
          const int sc = next.R.a.find(to.mq[mw]);
          if (sr < 0 || sc < 0 || next.L.a.sdim[sr] != S.kept[mk] || next.R.a.sdim[sc] != S.kept[mw]) continue;
          GemmTask task{};
          task.c_off = tn.base[mn] + tn.rowoff[mn][a] * tn.ncols[mn] + tn.coloff[mn][b];
          task.m = (int32_t)S.kept[mk];
          task.n = (int32_t)S.kept[mw];
          task.ldc = (int32_t)tn.ncols[mn];
          task.t0 = (int32_t)p.terms.size();
          GemmTerm tm{};
          tm.a_off = S.voff[mk] + to.coloff[mk][a];
          tm.lda = (int32_t)to.ncols[mk];
          tm.k = (int32_t)S.a2.sdim[t];
          tm.b_off = S.uoff[mw] + to.rowoff[mw][b] * S.kept[mw];
          tm.ldb = (int32_t)S.kept[mw];
          p.terms.push_back(tm);
          task.t1 = (int32_t)p.terms.size();
          p.tasks.push_back(task);
        }
      }
    if (!p.tasks.empty()) {
      status = p.validate(false, false, Vs.len, Us.len, tn.total, "prediction");
      if (status == CMPS_OK) status = p.upload(st);
      if (status == CMPS_OK) {
        cudaMemsetAsync(next.x.d, 0, sizeof(double) * 2 * tn.total, st);
        status = launch_zgemm_fp64(p, false, false, Vs, Us, next.x, st);
      }
      if (status == CMPS_OK && cudaStreamSynchronize(st) != cudaSuccess)
        status = fail(CMPS_ERR_CUDA, "prediction GEMM failed");
      if (status == CMPS_OK) *ok = true;
    }
  }
  p.release();
  Us.release();
  Vs.release();
  return status;
}

// MakeRFinitePrediction / MakeLFinitePrediction (DMRG_routines.cpp:709-716):
// the start vector of a sweep step.
//  moving right: theta'[(s2, a1), (s3, a3)] = sum_a2 (Lambda V^dagger)[a1, (s2, a2)] B[a2, (s3, a3)],
//                B = the right MPS tensor of the vertex entering the window (rsvd);
//  moving left:  theta'[(s0, a_), (s1, a1)] = sum_a0 A[(s0, a_), a0] (U Lambda)[(s1, a0), a1],
//                A = the left MPS tensor of the vertex entering the window (lsvd).
// One grouped FP64 GEMM from the sector blocks of the two factors into the new
// theta blocks; a block whose sectors do not line up is left out (zero).
int Dmrg::finite_predict(Heff& next, int dir, bool* ok) {
  *ok = false;
  if (!svd) return CMPS_OK;
  const int64_t nright = size - nleft - 2;
  auto& store_map = dir > 0 ? rsvd : lsvd;
  auto it = store_map.find(dir > 0 ? nright + 1 : nleft + 1);
  if (it == store_map.end() || !it->second) return CMPS_OK;
  const SvdResult& C = *svd;         // this window's factors (before the move)
  const SvdResult& O = *it->second;  // the stored tensor's factors
  cudaStream_t st = ctx->stream;
  const ThetaSpace& tc = C.th;
  const ThetaSpace& to = O.th;
  const ThetaSpace& tn = next.th;
  const Rules& r = next.rules;
  const int d = next.d;
  // Lambda on the current factor: rows of V^dagger (right) or columns of U (left)
  Planar S;
  const Planar& src = dir > 0 ? C.Vd : C.U;
  CMPS_TRY(S.alloc(std::max<int64_t>(1, src.len)));
  int status = CMPS_OK;
  for (int m = 0; m < (int)tc.mq.size() && status == CMPS_OK; ++m) {
    const int64_t k = C.kept[m];
    if (!k) continue;
    std::vector<double> lam(k);
    for (int64_t j = 0; j < k; ++j) lam[j] = lambda[C.gidx[m][j]];
    double* dl = nullptr;
    if (dmalloc(&dl, sizeof(double) * k) != cudaSuccess) {
      status = fail(CMPS_ERR_NOMEM, "finite prediction: scale allocation failed");
      break;
    }
    status = copy_wait(dl, lam.data(), sizeof(double) * k, cudaMemcpyHostToDevice, st);
    if (status == CMPS_OK) {
      if (dir > 0)
        k_scale_block<<<grid_n(k * tc.ncols[m]), 256, 0, st>>>(C.Vd.re() + C.voff[m], C.Vd.im() + C.voff[m], k,
                                                              tc.ncols[m], dl, nullptr, S.re() + C.voff[m],
                                                              S.im() + C.voff[m]);
      else
        k_scale_block<<<grid_n(tc.nrows[m] * k), 256, 0, st>>>(C.U.re() + C.uoff[m], C.U.im() + C.uoff[m],
                                                              tc.nrows[m], k, nullptr, dl, S.re() + C.uoff[m],
                                                              S.im() + C.uoff[m]);
      if (cudaStreamSynchronize(st) != cudaSuccess) status = fail(CMPS_ERR_CUDA, "finite prediction: scaling failed");
    }
    dfree(dl);
  }
  GemmPlan p;
  for (int mn = 0; mn < (int)tn.mq.size() && status == CMPS_OK; ++mn)
    for (int a = 0; a < d; ++a) {
      if (tn.rowoff[mn][a] < 0) continue;
      for (int b = 0; b < d; ++b) {
        if (tn.coloff[mn][b] < 0) continue;
        GemmTask task{};
        GemmTerm tm{};
        task.c_off = tn.base[mn] + tn.rowoff[mn][a] * tn.ncols[mn] + tn.coloff[mn][b];
        task.ldc = (int32_t)tn.ncols[mn];
        if (dir > 0) {
          // rows: new left bond sector q(mn) - q(a) = a current window block
          const int mc = tc.find(r.sub(tn.mq[mn], next.sigq[a]));
          if (mc < 0 || !C.kept[mc] || tc.coloff[mc][a] < 0) continue;
          const QKey t2 = r.add(tc.mq[mc], C.sigq[a]);  // a2 sector = the stored factor's block
          const int mo = to.find(t2);
          const int s2 = C.a2.find(t2);
          if (mo < 0 || s2 < 0 || O.kept[mo] != C.a2.sdim[s2] || to.coloff[mo][b] < 0) continue;
          const int sr = next.L.a.find(tc.mq[mc]);
          const int t3 = O.a2.find(r.add(t2, O.sigq[b]));
          const int sc = next.R.a.find(r.add(tn.mq[mn], next.sigq[b]));
          if (sr < 0 || t3 < 0 || sc < 0 || next.L.a.sdim[sr] != C.kept[mc] || next.R.a.sdim[sc] != O.a2.sdim[t3])
            continue;
          task.m = (int32_t)C.kept[mc];
          task.n = (int32_t)O.a2.sdim[t3];
          tm.a_off = C.voff[mc] + tc.coloff[mc][a];
          tm.lda = (int32_t)tc.ncols[mc];
          tm.k = (int32_t)O.kept[mo];
          tm.b_off = O.voff[mo] + to.coloff[mo][b];
          tm.ldb = (int32_t)to.ncols[mo];
        } else {
          // contraction over a0 of charge q(mn): the stored factor's block
          const int mo = to.find(tn.mq[mn]);
          if (mo < 0 || !O.kept[mo] || to.rowoff[mo][a] < 0) continue;
          const int mc = tc.find(r.add(tn.mq[mn], next.sigq[b]));
          if (mc < 0 || !C.kept[mc] || tc.rowoff[mc][b] < 0) continue;
          const int s0 = C.a0.find(tn.mq[mn]);
          if (s0 < 0 || C.a0.sdim[s0] != O.kept[mo]) continue;
          const int sr = next.L.a.find(r.sub(tn.mq[mn], next.sigq[a]));
          const int ro = O.a0.find(r.sub(tn.mq[mn], O.sigq[a]));
          const int sc = next.R.a.find(tc.mq[mc]);
          if (sr < 0 || ro < 0 || sc < 0 || next.L.a.sdim[sr] != O.a0.sdim[ro] || next.R.a.sdim[sc] != C.kept[mc])
            continue;
          task.m = (int32_t)O.a0.sdim[ro];
          task.n = (int32_t)C.kept[mc];
          tm.a_off = O.uoff[mo] + to.rowoff[mo][a] * O.kept[mo];
          tm.lda = (int32_t)O.kept[mo];
          tm.k = (int32_t)O.kept[mo];
          tm.b_off = C.uoff[mc] + tc.rowoff[mc][b] * C.kept[mc];
          tm.ldb = (int32_t)C.kept[mc];
        }
        task.t0 = (int32_t)p.terms.size();
        p.terms.push_back(tm);
        task.t1 = (int32_t)p.terms.size();
        p.tasks.push_back(task);
      }
    }
  if (status == CMPS_OK && !p.tasks.empty()) {
    const Planar& A = dir > 0 ? S : O.U;
    const Planar& B = dir > 0 ? O.Vd : S;
    status = p.validate(false, false, A.len, B.len, tn.total, "finite prediction");
    if (status == CMPS_OK) status = p.upload(st);
    if (status == CMPS_OK) {
      cudaMemsetAsync(next.x.d, 0, sizeof(double) * 2 * tn.total, st);
      status = launch_zgemm_fp64(p, false, false, A, B, next.x, st);
    }
    if (status == CMPS_OK && cudaStreamSynchronize(st) != cudaSuccess)
      status = fail(CMPS_ERR_CUDA, "finite prediction GEMM failed");
    if (status == CMPS_OK) *ok = true;
  }
  p.release();
  S.release();
  return status;
}

int Dmrg::step(int dir, int64_t chi, double trunc, double* out) {
  cudaStream_t st = ctx->stream;
  if (dir == 0 && !pstates.empty()) return fail(CMPS_ERR_STATE, "growth with projected states: the chain is finite");
  if (dir != 0) {
    if (!keep_blocks || !heff || !svd) return fail(CMPS_ERR_STATE, "finite sweep: grow with kept blocks first");
    const int64_t nright = size - nleft - 2;
    if (dir == 1 && nright < 1) return fail(CMPS_ERR_STATE, "finite sweep: already at the right end");
    if (dir == -1 && nleft < 1) return fail(CMPS_ERR_STATE, "finite sweep: already at the left end");
  }
  cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  struct EvGuard {
    cudaEvent_t* e;
    ~EvGuard() {
      for (int i = 0; i < 5; ++i)
        if (e[i]) cudaEventDestroy(e[i]);
    }
  } ev_guard{ev};
  for (auto& e : ev) CMPS_CUDA(cudaEventCreate(&e));
  using clock = std::chrono::steady_clock;
  auto ms_since = [](clock::time_point a, clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
  };
  const auto h0 = clock::now();
  cudaEventRecord(ev[0], st);
  Env L, R;
  if (dir == 1) {
    // MakeLeftBlock with A = U of this window; the right block of the new
    // window was stored by the growth or the previous sweep
    if (grad_on) CMPS_TRY(store_derivative(false, nleft + 1, st));
    Env nl;
    CMPS_TRY(left_update(*heff, *svd, nl));
    int rc = store(lblocks, nleft + 1, nl, st);
    nl.data.release();
    CMPS_TRY(rc);
    lsvd[nleft + 1] = svd;
    nleft += 1;
    auto ir = rblocks.find(size - nleft - 2);
    if (ir == rblocks.end()) return fail(CMPS_ERR_STATE, "finite sweep: right block missing");
    CMPS_TRY(copy_env(lblocks[nleft], L, st));
    CMPS_TRY(copy_env(ir->second, R, st));
    if (grad_on) CMPS_TRY(load_derivatives(nleft, size - nleft - 2, st));
  } else if (dir < 0) {
    if (grad_on) CMPS_TRY(store_derivative(true, size - nleft - 1, st));
    Env nr;
    CMPS_TRY(right_update(*heff, *svd, nr));
    int rc = store(rblocks, size - nleft - 1, nr, st);
    nr.data.release();
    CMPS_TRY(rc);
    rsvd[size - nleft - 1] = svd;
    nleft -= 1;
    auto il = lblocks.find(nleft);
    if (il == lblocks.end()) return fail(CMPS_ERR_STATE, "finite sweep: left block missing");
    CMPS_TRY(copy_env(il->second, L, st));
    CMPS_TRY(copy_env(rblocks[size - nleft - 2], R, st));
    if (grad_on) CMPS_TRY(load_derivatives(nleft, size - nleft - 2, st));
  } else if (dir == 2) {
    auto il = lblocks.find(nleft);
    auto ir = rblocks.find(size - nleft - 2);
    if (il == lblocks.end() || ir == rblocks.end()) return fail(CMPS_ERR_STATE, "window solve: a block is missing");
    CMPS_TRY(copy_env(il->second, L, st));
    CMPS_TRY(copy_env(ir->second, R, st));
  } else if (size == 0) {
    CMPS_TRY(dummy_blocks(L, R));
  } else {
    CMPS_TRY(left_update(*heff, *svd, L));
    CMPS_TRY(right_update(*heff, *svd, R));
    if (grad_on) {
      // derivative environments with the same truncation factors
      Env nl, nr;
      int rc = derivative_envs(*heff, *svd, dW, dl_ptr(), dr_ptr(), nl, nr);
      if (rc != CMPS_OK) {
        nl.data.release();
        nr.data.release();
        return rc;
      }
      dL.data.release();
      dR.data.release();
      dL = nl;
      dR = nr;
      have_dlr = true;
    }
  }
  if (dir == 0) {
    if (size > 0) nleft += 1;
    if (keep_blocks) {
      CMPS_TRY(store(lblocks, nleft, L, st));
      CMPS_TRY(store(rblocks, nleft, R, st));
      if (grad_on && dL.data.d) CMPS_TRY(store(dlblocks, nleft, dL, st));
      if (grad_on && dR.data.d) CMPS_TRY(store(drblocks, nleft, dR, st));
      if (svd) lsvd[nleft] = rsvd[nleft] = svd;  // the previous window's U and V^dagger made them
    }
  }
  cudaEventRecord(ev[4], st);
  const auto h_env = clock::now();
  auto next = std::unique_ptr<Heff>(new Heff());
  next->ctx = ctx;
  next->device = ctx->device;
  next->rules = rules;
  next->order_req = order_req;
  CMPS_TRY(next->parse_mpo(&W));
  if (grad_on) extend_pattern(next->W, dW);
  next->L = L;   // ownership of the device blocks moves to `next`
  next->R = R;
  CMPS_TRY(next->finish());
  const auto h_fin = clock::now();
  CMPS_TRY(prepare_precision(next.get(), precision));
  next->precision = precision;
  if (autotune) CMPS_TRY(next->autotune(&tune));
  const auto h_split = clock::now();
  bool have_guess = false;
  if (!pstates.empty())  // no prediction on excited-state steps (fDMRG_routines.cpp:118-121)
    CMPS_TRY(install_projectors(ctx, pstates, lsvd, rsvd, nleft, size, *next));
  else if (dir == 0) CMPS_TRY(predict(*next, &have_guess));
  else if (dir != 2) CMPS_TRY(finite_predict(*next, dir, &have_guess));
  const auto h_pred = clock::now();
  // the previous step's kept count per charge sizes this step's randomized SVD ranges
  std::map<QKey, int64_t> kept_hint;
  if (svd)
    for (size_t m = 0; m < svd->th.mq.size(); ++m) kept_hint[svd->th.mq[m]] = svd->kept[m];
  // the previous step's factors are released here unless a kept block needs them
  svd.reset();
  heff = std::move(next);
  const auto h_rel = clock::now();
  // a sweep step's fidelity compares the new state with the prediction the
  // eigensolve starts from, so keep a copy of it
  Planar guess;
  struct PlanarGuard {
    Planar* p;
    ~PlanarGuard() { p->release(); }
  } guess_guard{&guess};
  if (dir != 0 && want_fidelity && have_guess) {
    CMPS_TRY(guess.alloc(heff->th.total));
    CMPS_CUDA(cudaMemcpyAsync(guess.d, heff->x.d, sizeof(double) * 2 * heff->th.total, cudaMemcpyDeviceToDevice, st));
  }
  cudaEventRecord(ev[1], st);
  double e = 0.0;
  int nmv = 0;
  int rc = heff->eigs(nullptr, tol, restarts, kdim, &e, nullptr, &nmv, have_guess);
  if (rc != CMPS_OK && rc != CMPS_ERR_SOLVER) return rc;
  last_matvecs = nmv;
  last_grad = std::nan("");
  if (grad_on && rc == CMPS_OK)
    CMPS_TRY(heff_adjoint(*heff, dW, dl_ptr(), dr_ptr(), &last_grad));
  const auto h_eig = clock::now();
  cudaEventRecord(ev[2], st);
  svd = new_svd();
  // sweep steps next to an end keep every state up to chi (no weight cut),
  // as move_{right,left}_two_vertex do
  const int64_t nright_now = (dir == 0 ? size + 2 : size) - nleft - 2;
  const double cut = (dir == 1 && nright_now <= 1) || (dir == -1 && nleft <= 1) ? -0.0 : trunc;
  CMPS_TRY(theta_svd(*heff, chi, cut, *svd, kept_hint.empty() ? nullptr : &kept_hint));
  // SquareRescale(1.0) (MPS_matrix.hpp:66-70)
  std::vector<double> v = svd->values;
  double sq = 0.0;
  for (double x : v) sq += x * x;
  if (!(sq > 0.0)) return fail(CMPS_ERR_SOLVER, "square sum error: no weight kept");
  const double f = std::sqrt(1.0 / sq);
  for (double& x : v) x *= f;
  prev_lambda = size == 0 ? std::vector<double>(1, 1.0) : lambda;
  lambda = v;
  // growth steps report CheckConvergence, timed with the SVD phase
  double fid = std::nan("");
  if (dir == 0 && want_fidelity) CMPS_TRY(growth_fidelity(*heff, *svd, lambda, prev_lambda, &fid));
  if (dir != 0 && want_fidelity && guess.d) CMPS_TRY(sweep_fidelity(*heff, *svd, lambda, guess, &fid));
  cudaEventRecord(ev[3], st);
  cudaEventSynchronize(ev[3]);
  const auto h_svd = clock::now();
  float t01 = 0, t12 = 0, t23 = 0, t0e = 0;
  cudaEventElapsedTime(&t01, ev[0], ev[1]);
  cudaEventElapsedTime(&t12, ev[1], ev[2]);
  cudaEventElapsedTime(&t23, ev[2], ev[3]);
  cudaEventElapsedTime(&t0e, ev[0], ev[4]);
  last_ms[0] = t01;
  last_ms[1] = t12;
  last_ms[2] = t23;
  last_ms[3] = t01 + t12 + t23;
  const Heff::EigStats& es = heff->eig_stats;
  const double prof[kProfile] = {t0e,
                                 t01 - t0e,
                                 t12,
                                 t23,
                                 t01 + t12 + t23,
                                 (double)es.mv_split,
                                 (double)es.mv_fp64,
                                 (double)es.cycles,
                                 es.ms_split,
                                 es.ms_fp64,
                                 ms_since(h0, h_env),
                                 ms_since(h_env, h_fin),
                                 ms_since(h_fin, h_split),
                                 ms_since(h_split, h_pred),
                                 ms_since(h_pred, h_rel),
                                 ms_since(h_eig, h_svd),
                                 ms_since(h0, h_svd),
                                 (double)svd->routes[0],
                                 (double)svd->routes[1],
                                 (double)svd->routes[2],
                                 (double)heff->order};
  for (int i = 0; i < kProfile; ++i) last_profile[i] = prof[i];
  if (dir == 0) size += 2;
  out[0] = e;
  out[1] = e / (double)size;
  out[2] = entropy_of(lambda);
  out[3] = svd->discarded;
  out[4] = fid;
  return rc;
}

}  // namespace cmps

struct cmps_dmrg {
  std::unique_ptr<cmps::Dmrg> impl;
};

using namespace cmps;

extern "C" {

int cmps_dmrg_create(cmps_context* ctx, const cmps_charge_rules* rules, const cmps_mpx_desc* W,
                     const int16_t* target, int precision, cmps_dmrg** out) {
  if (!ctx || !rules || !W || !out) return fail(CMPS_ERR_ARG, "null argument");
  *out = nullptr;
  if (precision != CMPS_FP64 && !is_split(precision)) return fail(CMPS_ERR_ARG, "unknown precision");
  CMPS_CUDA(cudaSetDevice(ctx->device));
  auto d = std::unique_ptr<cmps_dmrg>(new cmps_dmrg());
  d->impl.reset(new Dmrg());
  Dmrg& D = *d->impl;
  D.ctx = ctx;
  D.device = ctx->device;
  if (rules->nq < 1 || rules->nq > kMaxQ) return fail(CMPS_ERR_ARG, "charge rules: bad count");
  D.rules.nq = rules->nq;
  for (int i = 0; i < rules->nq; ++i) D.rules.n[i] = rules->rules[i];
  D.precision = precision;
  // deep copy of W
  const int k = W->num_indices;
  if (k != 4) return fail(CMPS_ERR_ARG, "MPO: expected 4 indices");
  D.w_in.assign(W->inward, W->inward + k);
  D.w_ph.assign(W->physical, W->physical + k);
  D.w_sz.assign(W->sizes, W->sizes + k);
  int64_t nch = 0;
  for (int i = 0; i < k; ++i) nch += W->sizes[i];
  D.w_ch.assign(W->charges, W->charges + nch * rules->nq);
  D.w_cp.assign(W->colptr, W->colptr + W->cols + 1);
  const int64_t nnz = W->colptr[W->cols];
  D.w_ri.assign(W->rowind, W->rowind + nnz);
  D.w_val.assign(W->values, W->values + 2 * nnz);
  if (D.w_ri.empty()) {
    D.w_ri.push_back(0);
    D.w_val.push_back(0.0);
    D.w_val.push_back(0.0);
  }
  D.W = cmps_mpx_desc{4, W->num_row_indices, D.w_in.data(), D.w_ph.data(), D.w_sz.data(), D.w_ch.data(),
                      W->rows, W->cols, D.w_cp.data(), D.w_ri.data(), D.w_val.data()};
  Heff probe;
  probe.rules = D.rules;
  CMPS_TRY(probe.parse_mpo(&D.W));
  D.D = probe.D;
  D.bq = probe.bq;
  for (int c = 0; c < rules->nq; ++c) {
    int v = target ? target[c] : 0;
    if (D.rules.n[c] > 0) v = ((v % D.rules.n[c]) + D.rules.n[c]) % D.rules.n[c];
    D.target[c] = (int16_t)v;
  }
  *out = d.release();
  return CMPS_OK;
}

int cmps_dmrg_destroy(cmps_dmrg* d) {
  if (d && d->impl) cudaSetDevice(d->impl->device);
  delete d;
  cudaGetLastError();
  return CMPS_OK;
}

int cmps_dmrg_set_solver(cmps_dmrg* d, double tol, int max_restarts, int krylov_dim) {
  if (!d || !d->impl || !(tol > 0.0)) return fail(CMPS_ERR_ARG, "bad argument");
  d->impl->tol = tol;
  d->impl->restarts = max_restarts;
  d->impl->kdim = krylov_dim;
  return CMPS_OK;
}

static int dmrg_step(cmps_dmrg* d, int dir, int64_t chi, double max_trunc, double* row5, int64_t* bond_dim,
                     int* matvecs, double* ms4) {
  if (!d || !d->impl || !row5) return fail(CMPS_ERR_ARG, "null argument");
  Dmrg& D = *d->impl;
  CMPS_CUDA(cudaSetDevice(D.device));
  int rc = D.step(dir, chi, max_trunc, row5);
  if (bond_dim) *bond_dim = (int64_t)D.lambda.size();
  if (matvecs) *matvecs = D.last_matvecs;
  if (ms4)
    for (int i = 0; i < 4; ++i) ms4[i] = D.last_ms[i];
  return rc;
}

int cmps_dmrg_grow(cmps_dmrg* d, int64_t chi, double max_trunc, double* row5, int64_t* bond_dim, int* matvecs,
                   double* ms4) {
  return dmrg_step(d, 0, chi, max_trunc, row5, bond_dim, matvecs, ms4);
}

int cmps_dmrg_set_fidelity(cmps_dmrg* d, int on) {
  if (!d || !d->impl) return fail(CMPS_ERR_ARG, "null handle");
  d->impl->want_fidelity = on != 0;
  return CMPS_OK;
}

int cmps_dmrg_set_order(cmps_dmrg* d, int order) {
  if (!d || !d->impl) return fail(CMPS_ERR_ARG, "null handle");
  if (order != CMPS_ORDER_AUTO && order != CMPS_ORDER_FOLDED && order != CMPS_ORDER_CANONICAL)
    return fail(CMPS_ERR_ARG, "unknown contraction order");
  d->impl->order_req = order;
  return CMPS_OK;
}

int cmps_dmrg_set_autotune(cmps_dmrg* d, int on) {
  if (!d || !d->impl) return fail(CMPS_ERR_ARG, "null handle");
  d->impl->autotune = on != 0;
  return CMPS_OK;
}

int cmps_dmrg_autotune_stats(const cmps_dmrg* d, int* tuned, int* cached, double* ms_heuristic, double* ms_best) {
  if (!d || !d->impl) return fail(CMPS_ERR_ARG, "null handle");
  const TuneStats& s = d->impl->tune;
  if (tuned) *tuned = s.tuned;
  if (cached) *cached = s.cached;
  if (ms_heuristic) *ms_heuristic = s.ms_heuristic;
  if (ms_best) *ms_best = s.ms_best;
  return CMPS_OK;
}

int cmps_dmrg_keep_blocks(cmps_dmrg* d, int keep) {
  if (!d || !d->impl) return fail(CMPS_ERR_ARG, "null handle");
  if (d->impl->size != 0) return fail(CMPS_ERR_STATE, "choose block keeping before the first growth step");
  d->impl->keep_blocks = keep != 0;
  return CMPS_OK;
}

int cmps_dmrg_move(cmps_dmrg* d, int direction, int64_t chi, double max_trunc, double* row5, int64_t* bond_dim,
                   int* matvecs, double* ms4) {
  if (direction != 1 && direction != -1) return fail(CMPS_ERR_ARG, "direction must be +1 (right) or -1 (left)");
  return dmrg_step(d, direction, chi, max_trunc, row5, bond_dim, matvecs, ms4);
}

int cmps_dmrg_solve(cmps_dmrg* d, int64_t chi, double max_trunc, double* row5, int64_t* bond_dim, int* matvecs,
                    double* ms4) {
  return dmrg_step(d, 2, chi, max_trunc, row5, bond_dim, matvecs, ms4);
}

int cmps_dmrg_project_state(cmps_dmrg* d, double weight) {
  if (!d || !d->impl) return fail(CMPS_ERR_ARG, "null handle");
  if (!(weight >= 0.0)) return fail(CMPS_ERR_ARG, "projected state: weight must be non-negative");
  Dmrg& D = *d->impl;
  if (D.pstates.size() >= 64) return fail(CMPS_ERR_ARG, "projected state: at most 64 of them");
  CMPS_CUDA(cudaSetDevice(D.device));
  return D.project_state(weight);
}

int cmps_dmrg_projected_states(const cmps_dmrg* d, int* count) {
  if (!d || !d->impl || !count) return fail(CMPS_ERR_ARG, "null argument");
  *count = (int)d->impl->pstates.size();
  return CMPS_OK;
}

int cmps_dmrg_window_length(const cmps_dmrg* d, int64_t* n_allowed, int64_t* full_length) {
  if (!d || !d->impl) return fail(CMPS_ERR_ARG, "null handle");
  const Dmrg& D = *d->impl;
  if (!D.heff) return fail(CMPS_ERR_STATE, "no window");
  if (n_allowed) *n_allowed = D.heff->n_allowed;
  if (full_length) *full_length = D.heff->full_length;
  return CMPS_OK;
}

int cmps_dmrg_projector(const cmps_dmrg* d, int index, double* arpack_out) {
  if (!d || !d->impl || !arpack_out) return fail(CMPS_ERR_ARG, "null argument");
  const Dmrg& D = *d->impl;
  if (!D.heff) return fail(CMPS_ERR_STATE, "no window");
  Heff& H = *D.heff;
  if (index < 0 || index >= H.proj_np) return fail(CMPS_ERR_ARG, "projector index out of range");
  CMPS_CUDA(cudaSetDevice(D.device));
  cudaStream_t st = H.ctx->stream;
  Planar v;
  v.d = H.proj.d + 2 * H.th.total * index;
  v.len = H.th.total;
  const int rc = H.unpack(v, H.d_io, st);
  v.d = nullptr;
  CMPS_TRY(rc);
  const size_t n = (size_t)H.n_allowed;
  CMPS_CUDA(cudaMemcpyAsync(arpack_out, H.d_io, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, st));
  CMPS_CUDA(cudaStreamSynchronize(st));
  for (size_t i = 0; i < n; ++i) arpack_out[2 * i + 1] = -arpack_out[2 * i + 1];  // P = conj(phi)
  return CMPS_OK;
}

int cmps_dmrg_position(const cmps_dmrg* d, int64_t* nleft, int64_t* size) {
  if (!d || !d->impl) return fail(CMPS_ERR_ARG, "null handle");
  if (nleft) *nleft = d->impl->nleft;
  if (size) *size = d->impl->size;
  return CMPS_OK;
}

int cmps_dmrg_set_gradient(cmps_dmrg* d, const cmps_mpx_desc* dW) {
  if (!d || !d->impl) return fail(CMPS_ERR_ARG, "null handle");
  Dmrg& D = *d->impl;
  if (D.size != 0) return fail(CMPS_ERR_STATE, "set the gradient direction before the first growth step");
  CMPS_CUDA(cudaSetDevice(D.device));
  if (!dW) {
    D.grad_on = false;
    D.dW.clear();
    return CMPS_OK;
  }
  Heff ref;
  ref.rules = D.rules;
  CMPS_TRY(ref.parse_mpo(&D.W));
  CMPS_TRY(parse_derivative_mpo(ref, dW, D.dW));
  D.grad_on = true;
  return CMPS_OK;
}

int cmps_dmrg_gradient(const cmps_dmrg* d, double* grad) {
  if (!d || !d->impl || !grad) return fail(CMPS_ERR_ARG, "null argument");
  if (!d->impl->grad_on) return fail(CMPS_ERR_STATE, "no gradient direction set");
  *grad = d->impl->last_grad;
  return CMPS_OK;
}

int cmps_dmrg_profile(const cmps_dmrg* d, double* out, int n) {
  if (!d || !d->impl || !out || n < 0) return fail(CMPS_ERR_ARG, "null argument");
  for (int i = 0; i < n && i < Dmrg::kProfile; ++i) out[i] = d->impl->last_profile[i];
  return std::min(n, Dmrg::kProfile) == n ? CMPS_OK : fail(CMPS_ERR_ARG, "profile has 21 entries");
}

int cmps_dmrg_unit_cell(cmps_dmrg* d, double tol, int krylov_dim, double* out6) {
  if (!d || !d->impl || !out6) return fail(CMPS_ERR_ARG, "null argument");
  Dmrg& D = *d->impl;
  CMPS_CUDA(cudaSetDevice(D.device));
  if (!D.svd || !D.heff || D.prev_lambda.empty() || D.size < 4)
    return fail(CMPS_ERR_STATE, "unit cell: needs two growth steps or more");
  if (!(tol > 0.0)) return fail(CMPS_ERR_ARG, "unit cell: tolerance must be positive");
  UnitCellMeasure m;
  CMPS_TRY(unit_cell_measure(D.ctx, *D.svd, D.lambda, D.prev_lambda, D.heff->W, D.heff->D, tol, krylov_dim, &m));
  out6[0] = m.energy;
  out6[1] = m.entropy;
  out6[2] = m.eta_left;
  out6[3] = m.eta_right;
  out6[4] = (double)m.chi;
  out6[5] = m.energy_imag;
  return CMPS_OK;
}

int cmps_dmrg_values(const cmps_dmrg* d, double* values) {
  if (!d || !d->impl || !values) return fail(CMPS_ERR_ARG, "null argument");
  std::memcpy(values, d->impl->lambda.data(), sizeof(double) * d->impl->lambda.size());
  return CMPS_OK;
}

}  // extern "C"
