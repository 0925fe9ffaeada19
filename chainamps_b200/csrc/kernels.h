// FP64 vector kernels of the device Krylov solver (see kernels.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace cmps {

// Planar FP64 complex vectors of a fixed length n; reductions are two-pass
// (per-CTA partials, then a fixed-order reduction) so results are
// deterministic run to run.
struct VecOps {
  int64_t n = 0;
  int nb = 0;
  double* d_partial = nullptr;
  double* d_small = nullptr;
  int64_t* d_pidx = nullptr;
  int init(int64_t n);
  void release();
  // h[j] = <V_j, w> (conjugate-linear in V), k vectors with stride ldv; h_host gets 2k doubles.
  int multidot(const double* Vr, const double* Vi, int64_t ldv, int k, const double* wr, const double* wi,
               double* h_host, cudaStream_t st);
  // w += sign * sum_j h_j V_j
  int multiaxpy(const double* Vr, const double* Vi, int64_t ldv, int k, const double* h_host, double* wr,
                double* wi, double sign, cudaStream_t st);
  int norm2(const double* xr, const double* xi, double* out, cudaStream_t st);
  int scale_copy(const double* xr, const double* xi, double s, double* yr, double* yi, cudaStream_t st);
  int random(double* re, double* im, uint64_t seed, cudaStream_t st);
  // y = sum_j c_j V_j, c real
  int combine(const double* Vr, const double* Vi, int64_t ldv, int k, const double* c_host, double* yr,
              double* yi, cudaStream_t st);
  int absmax(const double* re, const double* im, double* val_sq, int64_t* idx, cudaStream_t st);

  // Krylov steps whose coefficients stay on the device (no host round trip).
  double* d_coef = nullptr;  // coefficient scratch, kCoefDoubles
  static constexpr int kCoefDoubles = 2048;
  // d_out[2j], d_out[2j+1] = <V_j, w> for j < k (k <= 128); d_out[2k] = |w|^2.
  int mdot_dev(const double* Vr, const double* Vi, int64_t ldv, int k, const double* wr, const double* wi,
               double* d_out, cudaStream_t st);
  // w -= sum_j h_j V_j with h = d_h (2k doubles); *d_nrm2 = |w|^2 afterwards.
  int maxpy_norm_dev(const double* Vr, const double* Vi, int64_t ldv, int k, const double* d_h, double* wr,
                     double* wi, double* d_nrm2, cudaStream_t st);
  // w -= c u (c = d_c[0] + i d_c[1]), then as mdot_dev with the updated w.
  int update_mdot_dev(const double* d_c, const double* ur, const double* ui, const double* Vr, const double* Vi,
                      int64_t ldv, int k, double* wr, double* wi, double* d_out, cudaStream_t st);
  // w -= (*d_beta) p (skipped when pr is null), then d_out[0..1] = <v, w>.
  int axpy_dot_dev(const double* pr, const double* pi, const double* d_beta, const double* vr, const double* vi,
                   double* wr, double* wi, double* d_out, cudaStream_t st);
  // alpha_j = *d_a1 + *d_a2, beta_j = sqrt(*d_nrm2), and the scale of the next
  // basis vector (0 when the Krylov space is exhausted).
  int lanczos_coef(const double* d_a1, const double* d_a2, const double* d_nrm2, int j, double* d_alpha,
                   double* d_beta, double* d_scale, cudaStream_t st);
  // y = s x with s = *d_s, or s = 1 / sqrt(*d_s) when inv_sqrt.
  int scale_dev(const double* xr, const double* xi, const double* d_s, bool inv_sqrt, double* yr, double* yi,
                cudaStream_t st);
  int phase_drop(double* re, double* im, double pr, double pi, double thr, cudaStream_t st);
};

}  // namespace cmps
