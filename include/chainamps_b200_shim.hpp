/* The reference's hot-path seams, kept with their signatures, over
 * libchainamps_b200.
 *
 * A maintainer of the reference adds this header to its build (the
 * reference's source directory on the include path, CXSparse's cs.h as for
 * the rest of the build) and forwards the bodies of its seams here, so that
 * iDMRG_DRV and fDMRG_DRV compile and run unchanged:
 *
 *   TwoVertexComponents::TwoVertexComponents (DMRG_routines.cpp:779-833)
 *       cmps_shim::attach(this);    -- the window goes to the GPU; LeftPart
 *                                      and RightPart are no longer formed
 *   TwoVertexComponents::~TwoVertexComponents
 *       cmps_shim::detach(this);
 *   TwoVertexMPOMPSMultiply (DMRG_routines.hpp:248, the ARPACK MV callback)
 *       cmps_shim::TwoVertexMPOMPSMultiply(t, in, out);
 *   TwoVertexComponents::HED (DMRG_routines.hpp:210)
 *       return cmps_shim::HED(*this, numevals, which, initial, converge);
 *   TwoVertexSVD / MPX_matrix::SVD (DMRG_routines.hpp:225, MPX_matrix.hpp:116)
 *       cmps_shim::SVD(components, theta, chi, truncation)
 *   MakeLeftBlock / MakeRightBlock (DMRG_routines.hpp:238-239)
 *       cmps_shim::MakeLeftBlock(components, chi, truncation) (and Right)
 *
 * Every function keeps the reference's error convention: a failure prints
 * the library's message and exits.  The reference's own definitions of the
 * functions replaced are removed from DMRG_routines.cpp (or compiled out).
 */
#ifndef CHAINAMPS_B200_SHIM_HPP
#define CHAINAMPS_B200_SHIM_HPP

#include <complex>
#include <map>
#include <memory>
#include <vector>

#include "DMRG_routines.hpp"  // the reference: TwoVertexComponents, MPX_matrix, MPS_matrix, ...
#include "chainamps_b200_shim_core.hpp"

namespace cmps_shim {

/* MPX_matrix keeps its number of row indices protected (MPX_matrix.hpp:65)
 * and has no accessor for it; a pointer to the member formed in a derived
 * class reads it from any MPX_matrix. */
struct MpxRowIndices : ajaj::MPX_matrix {
  static ajaj::MPXInt of(const ajaj::MPX_matrix& A) { return A.*(&MpxRowIndices::m_NumRowIndices); }
};

/* MPX_matrix -> Tensor: its indices (direction, physical flag, the charges
 * of every element) and its CSC matrix. */
inline Tensor to_tensor(const ajaj::MPX_matrix& A) {
  Tensor t;
  const ajaj::QNVector& rules = A.basis().getChargeRules();
  const std::vector<ajaj::MPXInt> dims = A.dimsvector();
  for (size_t i = 0; i < dims.size(); ++i) {
    const ajaj::MPXIndex& ix = A.Index((ajaj::Sparseint)i);
    t.inward.push_back(ix.Ingoing() ? 1 : 0);
    t.physical.push_back(ix.Physical() ? 1 : 0);
    t.sizes.push_back((int64_t)ix.size());
    for (ajaj::MPXInt e = 0; e < ix.size(); ++e) {
      ajaj::State s = ix.at(e);
      for (size_t q = 0; q < rules.size(); ++q) t.charges.push_back((int16_t)s[(ajaj::QuantumNumberInt)q]);
    }
  }
  t.num_row_indices = (int32_t)MpxRowIndices::of(A);
  ajaj::SparseMatrix M = const_cast<ajaj::MPX_matrix&>(A).matrix();  // a copy of the CSC array
  t.rows = M.rows();
  t.cols = M.cols();
  for (ajaj::Sparseint j = 0; j <= M.cols(); ++j) t.colptr.push_back(M.get_p(j));
  for (ajaj::Sparseint p = 0; p < M.get_p(M.cols()); ++p) {
    t.rowind.push_back(M.get_i(p));
    const std::complex<double> x = M.get_x(p);
    t.values.push_back(x.real());
    t.values.push_back(x.imag());
  }
  return t;
}

inline std::vector<int16_t> charge_rules(const ajaj::MPX_matrix& A) {
  const ajaj::QNVector& r = A.basis().getChargeRules();
  return std::vector<int16_t>(r.begin(), r.end());
}

/* One process-wide context on device 0 (the reference runs one host thread). */
inline Context& context() {
  static Context ctx(0);
  return ctx;
}

/* The device windows of live TwoVertexComponents objects. */
inline std::map<const ajaj::TwoVertexComponents*, std::unique_ptr<TwoVertex>>& registry() {
  static std::map<const ajaj::TwoVertexComponents*, std::unique_ptr<TwoVertex>> r;
  return r;
}

inline TwoVertex& attach(const ajaj::TwoVertexComponents* t, int precision = CMPS_FP64) {
  std::unique_ptr<TwoVertex>& slot = registry()[t];
  slot.reset(new TwoVertex(context(), charge_rules(t->H), to_tensor(t->LeftBlock), to_tensor(t->H),
                           to_tensor(t->RightBlock), precision));
  return *slot;
}

inline void detach(const ajaj::TwoVertexComponents* t) { registry().erase(t); }

inline TwoVertex& of(const ajaj::TwoVertexComponents* t) {
  auto it = registry().find(t);
  if (it == registry().end()) {
    std::printf("chainamps_b200: TwoVertexComponents not attached to the GPU\n");
    std::exit(1);
  }
  return *it->second;
}

/* TwoVertexMPOMPSMultiply (DMRG_routines.hpp:248): the ARPACK MV callback,
 * in and out being ARPACK's workd slices over allowed_indices. */
inline void TwoVertexMPOMPSMultiply(const ajaj::TwoVertexComponents* t, std::complex<double>* in,
                                    std::complex<double>* out) {
  two_vertex_multiply(&of(t), in, out);
}

/* TwoVertexComponents::HED (DMRG_routines.hpp:210) for the ground state
 * ("SR", one eigenpair), by the device's Krylov solver instead of ARPACK:
 * the same SparseHED (DMRG_routines.cpp:870-893), the eigenvector already
 * phase-fixed, dropped and FixComplexPrecision-ed by the library.  converge:
 * the reference's flag; the device solver always converges to tol. */
inline ajaj::SparseHED HED(const ajaj::TwoVertexComponents& t, ajaj::MPXInt numevals, char which[3],
                           const ajaj::SparseMatrix* initial = nullptr, bool converge = 1, double tol = 1e-10) {
  (void)converge;
  if (numevals != 1 || which[0] != 'S' || which[1] != 'R') {
    std::printf("chainamps_b200: HED computes the lowest eigenpair only (numevals 1, SR)\n");
    std::exit(1);
  }
  TwoVertex& g = of(&t);
  const size_t n = (size_t)g.size();
  std::vector<std::complex<double> > guess, evec(n);
  if (initial) {
    guess.resize(n);
    ajaj::SparseVectorWithRestriction gs(initial, &t.allowed_indices);
    ajaj::ConvertSparseVectorWithRestriction(&gs, guess.data());
  }
  const double e = g.lowest(initial ? guess.data() : nullptr, evec.data(), tol);
  ajaj::SparseHED ans(t.length(), 1);
  ans.Values.push_back(e);
  for (size_t i = 0; i < n; ++i)
    if (evec[i] != 0.0) ans.EigenVectors.entry(t.allowed_indices[i], 0, evec[i]);
  ans.EigenVectors.finalise();
  return ans;
}

/* A CSC matrix with interleaved values as the reference's SparseMatrix. */
inline ajaj::SparseMatrix to_sparse(int64_t rows, int64_t cols, const std::vector<int64_t>& colptr,
                                    const std::vector<int64_t>& rowind, const std::vector<double>& values) {
  ajaj::SparseMatrix M(rows, cols, (ajaj::Sparseint)(rowind.empty() ? 1 : rowind.size()));
  for (int64_t c = 0; c < cols; ++c)
    for (int64_t p = colptr[c]; p < colptr[c + 1]; ++p)
      M.entry(rowind[p], c, std::complex<double>(values[2 * p], values[2 * p + 1]));
  M.finalise();
  return M;
}

inline ajaj::StateArray states_of(const ajaj::MPX_matrix& basis_of, const std::vector<int16_t>& charges,
                                  int64_t count) {
  const ajaj::QNVector& rules = basis_of.basis().getChargeRules();
  ajaj::StateArray out;
  for (int64_t k = 0; k < count; ++k) {
    ajaj::QNVector v;
    for (size_t q = 0; q < rules.size(); ++q) v.push_back(charges[(size_t)k * rules.size() + q]);
    out.emplace_back(rules, v);
  }
  return out;
}

/* TwoVertexSVD / MPX_matrix::SVD (MPX_matrix.cpp:157-192) of the window's
 * last eigenvector (theta supplies the indices): U keeps theta's row indices
 * and gains the outgoing new bond, V^dagger the ingoing new bond and theta's
 * column indices; the new bond's charges come from the library in the kept
 * (descending) order. */
inline ajaj::MPXDecomposition SVD(const ajaj::TwoVertexComponents& t, const ajaj::MPX_matrix& theta,
                                  size_t bond_dimension, double truncation) {
  TwoVertex& g = of(&t);
  SvdFactors f = g.svd((int64_t)bond_dimension, truncation);
  ajaj::StateArray newstates = states_of(theta, f.new_charges, f.kept);
  const ajaj::MPXInt nrow = MpxRowIndices::of(theta);
  std::vector<ajaj::MPXIndex> left;
  for (ajaj::MPXInt i = 0; i < nrow; ++i) left.push_back(theta.Index(i));
  left.emplace_back(0, newstates);
  std::vector<ajaj::MPXIndex> right;
  right.emplace_back(1, newstates);
  const std::vector<ajaj::MPXInt> dims = theta.dimsvector();
  for (size_t i = (size_t)nrow; i < dims.size(); ++i) right.push_back(theta.Index((ajaj::Sparseint)i));
  return ajaj::MPXDecomposition(
      ajaj::MPX_matrix(theta.GetPhysicalSpectrum(), left, nrow,
                       to_sparse(g.theta_rows(), f.kept, f.u_colptr, f.u_rowind, f.u_values)),
      std::move(f.values),
      ajaj::MPX_matrix(theta.GetPhysicalSpectrum(), right, 1,
                       to_sparse(f.kept, g.theta_cols(), f.v_colptr, f.v_rowind, f.v_values)),
      f.discarded);
}

/* MakeLeftBlock / MakeRightBlock (DMRG_routines.cpp:594-611) for the next
 * window, from this window's environments and MPO and the U / V^dagger of
 * its SVD at (chi, truncation), in the reference's 6-index layouts: left
 * (a'_dummy, a', b_dummy, b, a_dummy, a), 3 row indices; right (a', a'_dummy,
 * b, b_dummy, a, a_dummy), 2 row indices. */
inline ajaj::MPX_matrix MakeBlock(const ajaj::TwoVertexComponents& t, size_t chi, double truncation, bool right) {
  TwoVertex& g = of(&t);
  BlockCSC b = right ? g.right_block((int64_t)chi, truncation) : g.left_block((int64_t)chi, truncation);
  const ajaj::MPX_matrix& H = t.H;
  ajaj::StateArray bond = states_of(H, b.a_charges, b.chi);
  ajaj::StateArray dummy(1, ajaj::State(H.basis().getChargeRules()));
  const ajaj::MPXIndex& bq = H.Index(right ? 3 : 1);  // the MPO bond the block carries
  std::vector<ajaj::MPXIndex> idx;
  if (!right) {
    idx.emplace_back(0, dummy);
    idx.emplace_back(1, bond);
    idx.emplace_back(1, dummy);
    idx.emplace_back(0, bq);
    idx.emplace_back(1, dummy);
    idx.emplace_back(0, bond);
  } else {
    idx.emplace_back(0, bond);
    idx.emplace_back(1, dummy);
    idx.emplace_back(1, bq);
    idx.emplace_back(0, dummy);
    idx.emplace_back(1, bond);
    idx.emplace_back(0, dummy);
  }
  return ajaj::MPX_matrix(H.basis(), idx, right ? 2 : 3,
                          to_sparse(b.chi, b.mpo_dim * b.chi, b.colptr, b.rowind, b.values));
}
inline ajaj::MPX_matrix MakeLeftBlock(const ajaj::TwoVertexComponents& t, size_t chi, double truncation) {
  return MakeBlock(t, chi, truncation, false);
}
inline ajaj::MPX_matrix MakeRightBlock(const ajaj::TwoVertexComponents& t, size_t chi, double truncation) {
  return MakeBlock(t, chi, truncation, true);
}

}  // namespace cmps_shim

#endif
