// Adjoint of the two-vertex H_eff contraction: the derivative of the
// variational energy E = <theta|H_eff|theta> / <theta|theta> with respect to
// a coupling lambda of the vertex MPO (an interchain coupling, a field),
// W(lambda) = W0 + lambda dW.
//
// H_eff is bilinear in the two vertex MPOs and linear in each environment:
//   H_eff theta = sum_b1 (LeftPart^{b1} theta) RightPart^{b1},
//   LeftPart  = sum_b0 W L^{b0},   RightPart = sum_b2 W R^{b2}.
// With the environments' own derivatives dL, dR (the same contraction with
// dW inserted at one earlier vertex, carried along by the environment
// update), the derivative of the contraction is
//   dH_eff theta = sum_b1 (LP_d^{b1} theta) RP^{b1} + (LP^{b1} theta) RP_d^{b1},
//   LP_d = LP(dL, W) + LP(L, dW),   RP_d = RP(dR, W) + RP(R, dW),
// so the gradient costs two FP64 matvecs through the same grouped-GEMM
// plans, with LP_d / RP_d formed in LeftPart / RightPart's own block layout.
// For the eigenvector theta, dE/dlambda = Re <theta|dH_eff|theta> / <theta|theta>
// (Hellmann-Feynman; the truncation bases of earlier steps are held fixed).
//
// There is no reference counterpart: ChainAMPS has no derivative path.
#include <cuda_runtime.h>

#include <map>
#include <set>
#include <vector>

#include "heff.h"

namespace cmps {

static bool same_layout(const Env& a, const Env& b) {
  return a.right == b.right && a.D == b.D && a.a.size() == b.a.size() && a.off == b.off && a.data.len == b.data.len;
}

// Blocks and terms of LP(L, dW) (left) or RP(R, dW) (right) in the layout of
// H's LeftPart / RightPart; fails when dW has an entry that W lacks.
static int dw_terms(const Heff& H, const std::vector<WEntry>& dW, bool right, std::vector<AxpyBlock>& blocks,
                    std::vector<AxpyTerm>& terms) {
  const Rules& r = H.rules;
  const ThetaSpace& th = H.th;
  const Bond& A = right ? H.R.a : H.L.a;
  const Env& E = right ? H.R : H.L;
  const auto& off = right ? H.rp_off : H.lp_off;
  std::map<std::array<int, 4>, std::vector<AxpyTerm>> per;
  for (const WEntry& w : dW) {
    for (int s = 0; s < A.nsec(); ++s) {
      const int b_env = right ? w.br : w.bl;
      const int64_t o = E.off[(size_t)b_env * A.nsec() + s];
      if (o < 0) continue;
      if (!right) {
        QKey m = r.add(H.sigq[w.s], A.sq[s]);
        if (th.find(m) < 0 || th.find(r.add(m, H.bq[w.br])) < 0) continue;
        per[{w.br, w.sp, w.s, s}].push_back(AxpyTerm{o, w.wr, w.wi});
      } else {
        QKey m = r.sub(A.sq[s], H.sigq[w.s]);
        if (th.find(m) < 0 || th.find(r.add(m, H.bq[w.bl])) < 0) continue;
        per[{w.bl, w.s, w.sp, s}].push_back(AxpyTerm{o, w.wr, w.wi});
      }
    }
  }
  blocks.clear();
  terms.clear();
  for (auto& kv : per) {
    auto it = off.find(kv.first);
    if (it == off.end()) return fail(CMPS_ERR_ARG, "adjoint: dW has an entry outside the pattern of W");
    const auto& key = kv.first;
    const int s = key[3];
    // partner sector, as in Heff::finish
    QKey qp = r.sub(r.add(r.add(A.sq[s], H.sigq[key[2]]), H.bq[key[0]]), H.sigq[key[1]]);
    const int sp = A.find(qp);
    if (sp < 0) return fail(CMPS_ERR_STATE, "adjoint: partner sector missing");
    const int64_t len = A.sdim[sp] * A.sdim[s];
    blocks.push_back(AxpyBlock{it->second, len, (int32_t)terms.size(), (int32_t)(terms.size() + kv.second.size())});
    for (auto& t : kv.second) terms.push_back(t);
  }
  return CMPS_OK;
}

int derivative_parts(Heff& H, const std::vector<WEntry>& dW, const Env* dL, const Env* dR, Planar& LPd,
                     Planar& RPd) {
  if (dL && !same_layout(*dL, H.L)) return fail(CMPS_ERR_ARG, "adjoint: dL has a different block layout from L");
  if (dR && !same_layout(*dR, H.R)) return fail(CMPS_ERR_ARG, "adjoint: dR has a different block layout from R");
  cudaStream_t st = H.ctx->stream;
  CMPS_TRY(LPd.alloc(H.LP.len));
  CMPS_TRY(RPd.alloc(H.RP.len));
  CMPS_TRY(zero_wait(LPd.d, sizeof(double) * 2 * LPd.len, st));
  CMPS_TRY(zero_wait(RPd.d, sizeof(double) * 2 * RPd.len, st));
  // environment parts: the matvec's own block lists with dL / dR as source
  if (dL) CMPS_TRY(launch_block_axpy(H.d_lp_blocks, (int)H.lp_blocks.size(), H.d_lp_terms, dL->data, LPd, st, true));
  if (dR) CMPS_TRY(launch_block_axpy(H.d_rp_blocks, (int)H.rp_blocks.size(), H.d_rp_terms, dR->data, RPd, st, true));
  // vertex parts: dW in place of W
  for (int side = 0; side < 2; ++side) {
    std::vector<AxpyBlock> blocks;
    std::vector<AxpyTerm> terms;
    CMPS_TRY(dw_terms(H, dW, side == 1, blocks, terms));
    if (blocks.empty()) continue;
    AxpyBlock* db = nullptr;
    AxpyTerm* dt = nullptr;
    int rc = CMPS_OK;
    if (dmalloc(&db, sizeof(AxpyBlock) * blocks.size()) != cudaSuccess ||
        dmalloc(&dt, sizeof(AxpyTerm) * terms.size()) != cudaSuccess)
      rc = fail(CMPS_ERR_NOMEM, "adjoint: term list allocation failed");
    if (rc == CMPS_OK) rc = copy_wait(db, blocks.data(), sizeof(AxpyBlock) * blocks.size(), cudaMemcpyHostToDevice, st);
    if (rc == CMPS_OK) rc = copy_wait(dt, terms.data(), sizeof(AxpyTerm) * terms.size(), cudaMemcpyHostToDevice, st);
    if (rc == CMPS_OK)
      rc = launch_block_axpy(db, (int)blocks.size(), dt, side == 0 ? H.L.data : H.R.data, side == 0 ? LPd : RPd, st,
                             true);
    if (rc == CMPS_OK && cudaStreamSynchronize(st) != cudaSuccess)
      rc = fail(CMPS_ERR_CUDA, "adjoint: LeftPart/RightPart derivative failed");
    dfree(db);
    dfree(dt);
    CMPS_TRY(rc);
  }
  return CMPS_OK;
}

int parse_derivative_mpo(const Heff& H, const cmps_mpx_desc* dW, std::vector<WEntry>& out) {
  Heff tmp;
  tmp.rules = H.rules;
  CMPS_TRY(tmp.parse_mpo(dW));
  if (tmp.d != H.d || tmp.D != H.D || tmp.sigq != H.sigq || tmp.bq != H.bq)
    return fail(CMPS_ERR_ARG, "adjoint: dW indices differ from the MPO's");
  out = tmp.W;
  return CMPS_OK;
}

void extend_pattern(std::vector<WEntry>& W, const std::vector<WEntry>& dW) {
  std::set<std::array<int, 4>> have;
  for (const WEntry& w : W) have.insert({w.sp, w.bl, w.s, w.br});
  for (const WEntry& w : dW)
    if (have.insert({w.sp, w.bl, w.s, w.br}).second) W.push_back(WEntry{w.sp, w.bl, w.s, w.br, 0.0, 0.0});
}

int heff_adjoint(Heff& H, const std::vector<WEntry>& dW, const Env* dL, const Env* dR, double* grad) {
  if (!H.have_theta) return fail(CMPS_ERR_STATE, "adjoint: no wavefunction (call cmps_heff_eigs or cmps_heff_set_theta)");
  if (!H.whole()) return fail(CMPS_ERR_STATE, "adjoint: the matvec is sharded");
  cudaStream_t st = H.ctx->stream;
  Planar LPd, RPd;
  int rc = derivative_parts(H, dW, dL, dR, LPd, RPd);
  double* d_out = H.ops.d_coef + 1024;  // 2 x 3 doubles, clear of the Lanczos coefficients
  double h[6] = {0, 0, 0, 0, 0, 0};
  if (rc == CMPS_OK) {
    // <theta| (LP_d theta) RP >
    std::swap(H.LP, LPd);
    rc = H.apply_folded_fp64(H.theta, H.y, st);
    std::swap(H.LP, LPd);
  }
  if (rc == CMPS_OK) rc = H.ops.mdot_dev(H.theta.re(), H.theta.im(), 0, 1, H.y.re(), H.y.im(), d_out, st);
  if (rc == CMPS_OK) {
    // <theta| (LP theta) RP_d >
    std::swap(H.RP, RPd);
    rc = H.apply_folded_fp64(H.theta, H.y, st);
    std::swap(H.RP, RPd);
  }
  if (rc == CMPS_OK) rc = H.ops.mdot_dev(H.theta.re(), H.theta.im(), 0, 1, H.y.re(), H.y.im(), d_out + 3, st);
  if (rc == CMPS_OK) rc = copy_wait(h, d_out, sizeof(double) * 6, cudaMemcpyDeviceToHost, st);
  double nrm = 0.0;
  if (rc == CMPS_OK) rc = H.ops.norm2(H.theta.re(), H.theta.im(), &nrm, st);
  LPd.release();
  RPd.release();
  CMPS_TRY(rc);
  if (!(nrm > 0.0)) return fail(CMPS_ERR_STATE, "adjoint: zero wavefunction");
  *grad = (h[0] + h[3]) / nrm;
  return CMPS_OK;
}

// The derivative environments of the next step: the environment update with
// LeftPart / RightPart replaced by their derivatives (the truncation factors
// U, V^dagger of this step held fixed).
int derivative_envs(Heff& H, const SvdResult& s, const std::vector<WEntry>& dW, const Env* dL, const Env* dR,
                    Env& dLn, Env& dRn) {
  Planar LPd, RPd;
  int rc = derivative_parts(H, dW, dL, dR, LPd, RPd);
  if (rc == CMPS_OK) {
    std::swap(H.LP, LPd);
    rc = left_update(H, s, dLn);
    std::swap(H.LP, LPd);
  }
  if (rc == CMPS_OK) {
    std::swap(H.RP, RPd);
    rc = right_update(H, s, dRn);
    std::swap(H.RP, RPd);
  }
  LPd.release();
  RPd.release();
  return rc;
}

}  // namespace cmps

using namespace cmps;

extern "C" int cmps_heff_adjoint(cmps_heff* h, const cmps_mpx_desc* dW, const cmps_block* dL, const cmps_block* dR,
                                 double* grad) {
  if (!h || !h->impl || !dW || !grad) return fail(CMPS_ERR_ARG, "null argument");
  Heff& H = *h->impl;
  CMPS_CUDA(cudaSetDevice(H.device));
  cudaGetLastError();
  std::vector<WEntry> w;
  CMPS_TRY(parse_derivative_mpo(H, dW, w));
  return heff_adjoint(H, w, dL ? &dL->env : nullptr, dR ? &dR->env : nullptr, grad);
}
