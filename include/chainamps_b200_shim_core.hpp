/* C++ layer over the C ABI of libchainamps_b200 (include/chainamps_b200.h),
 * independent of the reference's classes.
 *
 * It gives the reference's hot-path seams their C++ shape -- RAII handles,
 * std::complex<double> host vectors in ARPACK order, and the error
 * convention of printing the message and exiting (the reference has no
 * exceptions) -- so that include/chainamps_b200_shim.hpp only has to turn
 * the reference's own objects (MPX_matrix, TwoVertexComponents) into
 * Tensors and back.
 *
 *   cmps_shim::TwoVertex          TwoVertexComponents (DMRG_routines.hpp:189-214)
 *   two_vertex_multiply(t, in, out)
 *                                 TwoVertexMPOMPSMultiply (DMRG_routines.hpp:248),
 *                                 the MV callback ARPACK's reverse-communication
 *                                 loop calls (arpack_interface.hpp:243-247)
 *   TwoVertex::lowest             TwoVertexComponents::HED (DMRG_routines.hpp:210)
 *   TwoVertex::svd / SvdFactors   MPX_matrix::SVD (MPX_matrix.hpp:116)
 *   TwoVertex::left_block / right_block
 *                                 MakeLeftBlock / MakeRightBlock
 *                                 (DMRG_routines.hpp:238-239)
 *   load_tensor / store_tensor    load_MPX_matrix / MPX_matrix::store
 *                                 (MPX_matrix.cpp:219-247, 593-607)
 */
#ifndef CHAINAMPS_B200_SHIM_CORE_HPP
#define CHAINAMPS_B200_SHIM_CORE_HPP

#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "chainamps_b200.h"

namespace cmps_shim {

/* The reference's error convention: print the library's message and exit(1). */
inline void check(int status) {
  if (status != CMPS_OK) {
    std::printf("chainamps_b200: %s\n", cmps_last_error());
    std::fflush(stdout);
    std::exit(1);
  }
}

/* One MPX_matrix as the C ABI takes it (MPX_matrix.hpp:61-66): directed,
 * charge-labelled indices, the number of row indices, one CSC matrix with the
 * first index fastest.  values are interleaved (re, im). */
struct Tensor {
  std::vector<uint8_t> inward, physical;
  std::vector<int64_t> sizes;
  std::vector<int16_t> charges;  // (sum of sizes) x nq
  int32_t num_row_indices = 0;
  int64_t rows = 0, cols = 0;
  std::vector<int64_t> colptr, rowind;
  std::vector<double> values;
  cmps_mpx_desc desc() const {
    cmps_mpx_desc d;
    d.num_indices = (int32_t)sizes.size();
    d.num_row_indices = num_row_indices;
    d.inward = inward.data();
    d.physical = physical.data();
    d.sizes = sizes.data();
    d.charges = charges.data();
    d.rows = rows;
    d.cols = cols;
    d.colptr = colptr.data();
    d.rowind = rowind.data();
    d.values = values.data();
    return d;
  }
};

/* A tensor read from the reference's binary MPX_matrix file; physical
 * indices take basis_charges (basis_size x nq). */
inline Tensor load_tensor(const std::string& path, int32_t nq, const std::vector<int16_t>& basis_charges = {}) {
  int32_t ni = 0, nr = 0;
  int64_t total = 0, rows = 0, cols = 0, nnz = 0;
  check(cmps_mpx_stat(path.c_str(), nq, &ni, &nr, &total, &rows, &cols, &nnz));
  Tensor t;
  t.inward.resize(ni);
  t.physical.resize(ni);
  t.sizes.resize(ni);
  t.charges.resize((size_t)total * nq);
  t.num_row_indices = nr;
  t.rows = rows;
  t.cols = cols;
  t.colptr.resize(cols + 1);
  t.rowind.resize(nnz > 0 ? nnz : 1);
  t.values.resize(2 * (nnz > 0 ? nnz : 1));
  check(cmps_mpx_load(path.c_str(), nq, basis_charges.empty() ? nullptr : basis_charges.data(),
                      (int64_t)(basis_charges.size() / (nq > 0 ? nq : 1)), t.inward.data(), t.physical.data(),
                      t.sizes.data(), t.charges.data(), t.colptr.data(), t.rowind.data(), t.values.data()));
  t.rowind.resize(nnz);
  t.values.resize(2 * nnz);
  return t;
}

inline void store_tensor(const Tensor& t, int32_t nq, const std::string& path) {
  cmps_mpx_desc d = t.desc();
  check(cmps_mpx_store(&d, nq, path.c_str()));
}

/* One device and its stream (cmps_context). */
class Context {
 public:
  explicit Context(int device = 0) { check(cmps_context_create(device, &c_)); }
  ~Context() { cmps_context_destroy(c_); }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;
  cmps_context* get() const { return c_; }

 private:
  cmps_context* c_ = nullptr;
};

/* The block SVD of the window's wavefunction (cmps_svd), copied to the host:
 * the kept values, the new bond's charges, U ((d chiL) x kept) and
 * V^dagger (kept x (d chiR)) in CSC with interleaved complex values. */
struct SvdFactors {
  int64_t kept = 0;
  double discarded = 0.0;
  std::vector<double> values;
  std::vector<int16_t> new_charges;  // kept x nq
  std::vector<int64_t> u_colptr, u_rowind, v_colptr, v_rowind;
  std::vector<double> u_values, v_values;
};

/* A device block (cmps_block) exported in the reference's 6-index layout:
 * rows a', columns b + D a (MakeLeftBlock / MakeRightBlock). */
struct BlockCSC {
  int64_t chi = 0, mpo_dim = 0;
  std::vector<int16_t> a_charges;  // chi x nq
  std::vector<int64_t> colptr, rowind;
  std::vector<double> values;
};

/* One two-vertex window on the device: the environments L and R and the MPO
 * W of the reference's TwoVertexComponents, as charge-sector blocks. */
class TwoVertex {
 public:
  TwoVertex(Context& ctx, const std::vector<int16_t>& rules, const Tensor& L, const Tensor& W, const Tensor& R,
            int precision = CMPS_FP64)
      : rules_(rules) {
    cmps_charge_rules cr;
    cr.nq = (int32_t)rules_.size();
    cr.rules = rules_.data();
    cmps_mpx_desc l = L.desc(), w = W.desc(), r = R.desc();
    check(cmps_heff_create(ctx.get(), &cr, &l, &w, &r, precision, &h_));
    check(cmps_heff_length(h_, &n_, &full_));
    // theta as a matrix: rows (sigma1, a0), columns (sigma2, a2); the left
    // block's a is index 5, the right block's a is index 4
    // (MakeLeftBlock / MakeRightBlock layouts), sigma is the MPO's index 0
    vrows_ = W.sizes.at(0) * L.sizes.at(5);
    vcols_ = W.sizes.at(0) * R.sizes.at(4);
  }
  ~TwoVertex() { cmps_heff_destroy(h_); }
  TwoVertex(const TwoVertex&) = delete;
  TwoVertex& operator=(const TwoVertex&) = delete;

  cmps_heff* handle() const { return h_; }
  int64_t size() const { return n_; }           // allowed_indices.size()
  int64_t length() const { return full_; }      // TwoVertexComponents::length()
  int32_t num_charges() const { return (int32_t)rules_.size(); }
  std::vector<int64_t> allowed_indices() const {
    std::vector<int64_t> a((size_t)n_);
    check(cmps_heff_allowed_indices(h_, a.data()));
    return a;
  }
  /* H_eff . in over the allowed entries: host arrays of size() complex values. */
  void multiply(const std::complex<double>* in, std::complex<double>* out) const {
    check(cmps_heff_apply(h_, reinterpret_cast<const double*>(in), reinterpret_cast<double*>(out)));
  }
  /* Lowest eigenpair (HED with numevals 1, "SR"): returns the eigenvalue; evec
   * (size() values, may be null) gets the vector after HED's phase fix, drop
   * and FixComplexPrecision (DMRG_routines.cpp:870-889).  guess may be null. */
  double lowest(const std::complex<double>* guess, std::complex<double>* evec, double tol = 1e-10,
                int* matvecs = nullptr, int max_restarts = 50, int krylov_dim = 24) {
    double e = 0.0;
    int nmv = 0;
    check(cmps_heff_eigs(h_, reinterpret_cast<const double*>(guess), tol, max_restarts, krylov_dim, &e,
                         reinterpret_cast<double*>(evec), &nmv));
    if (matvecs) *matvecs = nmv;
    return e;
  }
  /* Block SVD of the last eigenvector, with the reference's truncation rule
   * (bond dimension cap, discarded-weight cut, 1e-3 degeneracy extension). */
  SvdFactors svd(int64_t chi, double max_trunc) const {
    cmps_svd* s = nullptr;
    check(cmps_heff_theta_svd(h_, chi, max_trunc, &s));
    SvdFactors f;
    int64_t nnzu = 0, nnzv = 0;
    check(cmps_svd_info(s, &f.kept, &f.discarded, &nnzu, &nnzv));
    f.values.resize((size_t)f.kept);
    f.new_charges.resize((size_t)f.kept * rules_.size());
    f.u_colptr.resize((size_t)f.kept + 1);
    f.u_rowind.resize((size_t)(nnzu > 0 ? nnzu : 1));
    f.u_values.resize((size_t)(2 * (nnzu > 0 ? nnzu : 1)));
    f.v_colptr.resize((size_t)vcols_ + 1);
    f.v_rowind.resize((size_t)(nnzv > 0 ? nnzv : 1));
    f.v_values.resize((size_t)(2 * (nnzv > 0 ? nnzv : 1)));
    check(cmps_svd_copy(s, f.values.data(), f.new_charges.data(), f.u_colptr.data(), f.u_rowind.data(),
                        f.u_values.data(), f.v_colptr.data(), f.v_rowind.data(), f.v_values.data()));
    cmps_svd_destroy(s);
    f.u_rowind.resize((size_t)nnzu);
    f.u_values.resize((size_t)(2 * nnzu));
    f.v_rowind.resize((size_t)nnzv);
    f.v_values.resize((size_t)(2 * nnzv));
    return f;
  }
  /* MakeLeftBlock / MakeRightBlock from this window's environments, MPO and
   * the U / V^dagger of its SVD at (chi, max_trunc). */
  BlockCSC left_block(int64_t chi, double max_trunc) const { return block(chi, max_trunc, false); }
  BlockCSC right_block(int64_t chi, double max_trunc) const { return block(chi, max_trunc, true); }
  int64_t theta_rows() const { return vrows_; }
  int64_t theta_cols() const { return vcols_; }

 private:
  BlockCSC block(int64_t chi, double max_trunc, bool right) const {
    cmps_svd* s = nullptr;
    check(cmps_heff_theta_svd(h_, chi, max_trunc, &s));
    cmps_block* b = nullptr;
    check(right ? cmps_heff_right_block(h_, s, &b) : cmps_heff_left_block(h_, s, &b));
    cmps_svd_destroy(s);
    BlockCSC out;
    int64_t nnz = 0;
    check(cmps_block_info(b, &out.chi, &out.mpo_dim, &nnz));
    out.a_charges.resize((size_t)out.chi * rules_.size());
    out.colptr.resize((size_t)(out.mpo_dim * out.chi + 1));
    out.rowind.resize((size_t)(nnz > 0 ? nnz : 1));
    out.values.resize((size_t)(2 * (nnz > 0 ? nnz : 1)));
    check(cmps_block_copy(b, out.a_charges.data(), out.colptr.data(), out.rowind.data(), out.values.data()));
    cmps_block_destroy(b);
    out.rowind.resize((size_t)nnz);
    out.values.resize((size_t)(2 * nnz));
    return out;
  }

  std::vector<int16_t> rules_;
  cmps_heff* h_ = nullptr;
  int64_t n_ = 0, full_ = 0, vrows_ = 0, vcols_ = 0;
};

/* The ARPACK MV callback shape of TwoVertexMPOMPSMultiply
 * (DMRG_routines.hpp:248): in and out are slices of ARPACK's workd, valid for
 * the call, size() complex values each. */
inline void two_vertex_multiply(const TwoVertex* t, std::complex<double>* in, std::complex<double>* out) {
  t->multiply(in, out);
}

}  // namespace cmps_shim

#endif
