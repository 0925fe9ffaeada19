// Memory-bound kernels of the hot path: block AXPY lists (LeftPart /
// RightPart formation) and the FP64 vector kernels of the device Krylov
// solver.  All are grid-stride loops sized to a multiple of the SM count.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "internal.h"
#include "kernels.h"

namespace cmps {

namespace {

int grid_for(int64_t n, int threads) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int64_t want = (n + threads - 1) / threads;
  int64_t cap = (int64_t)sms * 8;
  if (want < 1) want = 1;
  return (int)(want < cap ? want : cap);
}

// One CTA per destination block; dst = sum_t w_t src_t (dst += ... when
// `accumulate`).
__global__ void k_block_axpy(const AxpyBlock* __restrict__ blocks, const AxpyTerm* __restrict__ terms,
                             const double* __restrict__ sr, const double* __restrict__ si,
                             double* __restrict__ dr, double* __restrict__ di, int accumulate) {
  const AxpyBlock b = blocks[blockIdx.x];
  for (int64_t e = threadIdx.x; e < b.len; e += blockDim.x) {
    double xr = 0.0, xi = 0.0;
    for (int t = b.t0; t < b.t1; ++t) {
      const AxpyTerm tm = terms[t];
      double vr = sr[tm.src_off + e], vi = si[tm.src_off + e];
      xr += tm.wr * vr - tm.wi * vi;
      xi += tm.wr * vi + tm.wi * vr;
    }
    if (accumulate) {
      xr += dr[b.dst_off + e];
      xi += di[b.dst_off + e];
    }
    dr[b.dst_off + e] = xr;
    di[b.dst_off + e] = xi;
  }
}

// ---- Krylov vector kernels (planar FP64 vectors of length n) ----------------
constexpr int RED_THREADS = 256;

// partial[j][blk] = sum_i conj(V_j[i]) * w[i] over this CTA's slice, j < k.
__global__ void k_multidot(const double* __restrict__ Vr, const double* __restrict__ Vi, int64_t ldv,
                           int k, const double* __restrict__ wr, const double* __restrict__ wi, int64_t n,
                           double* __restrict__ partial) {
  extern __shared__ double red[];
  for (int j = 0; j < k; ++j) {
    double sr = 0.0, si = 0.0;
    const double* vr = Vr + (int64_t)j * ldv;
    const double* vi = Vi + (int64_t)j * ldv;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      double ar = vr[i], ai = vi[i], br = wr[i], bi = wi[i];
      sr += ar * br + ai * bi;
      si += ar * bi - ai * br;
    }
    red[threadIdx.x] = sr;
    red[threadIdx.x + blockDim.x] = si;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) {
        red[threadIdx.x] += red[threadIdx.x + s];
        red[threadIdx.x + blockDim.x] += red[threadIdx.x + s + blockDim.x];
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      partial[(2 * j) * gridDim.x + blockIdx.x] = red[0];
      partial[(2 * j + 1) * gridDim.x + blockIdx.x] = red[blockDim.x];
    }
    __syncthreads();
  }
}

// out[r] = sum_b partial[r][b], r < rows (one warp-per-row, deterministic order).
__global__ void k_reduce_rows(const double* __restrict__ partial, int nb, int rows, double* __restrict__ out) {
  int r = blockIdx.x;
  if (r >= rows) return;
  __shared__ double red[RED_THREADS];
  double s = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partial[(int64_t)r * nb + b];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[r] = red[0];
}

// w -= sum_j h_j V_j  (h complex, k <= 64 in constant-like global memory)
__global__ void k_multiaxpy(const double* __restrict__ Vr, const double* __restrict__ Vi, int64_t ldv, int k,
                            const double* __restrict__ h, double* __restrict__ wr, double* __restrict__ wi,
                            int64_t n, double sign) {
  __shared__ double hs[2 * 128];
  for (int j = threadIdx.x; j < 2 * k; j += blockDim.x) hs[j] = h[j];
  __syncthreads();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double xr = 0.0, xi = 0.0;
    for (int j = 0; j < k; ++j) {
      double hr = hs[2 * j], hi = hs[2 * j + 1];
      double vr = Vr[(int64_t)j * ldv + i], vi = Vi[(int64_t)j * ldv + i];
      xr += hr * vr - hi * vi;
      xi += hr * vi + hi * vr;
    }
    wr[i] += sign * xr;
    wi[i] += sign * xi;
  }
}

__global__ void k_scale_copy(const double* __restrict__ xr, const double* __restrict__ xi, double s,
                             double* __restrict__ yr, double* __restrict__ yi, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    yr[i] = s * xr[i];
    yi[i] = s * xi[i];
  }
}

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdULL;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ULL;
  x ^= x >> 33;
  return x;
}

__global__ void k_random(double* __restrict__ re, double* __restrict__ im, int64_t n, uint64_t seed) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t a = mix64(seed ^ (2 * (uint64_t)i + 1));
    uint64_t b = mix64(a + 0x9e3779b97f4a7c15ULL);
    re[i] = ((double)(a >> 11) * (1.0 / 9007199254740992.0)) - 0.5;
    im[i] = ((double)(b >> 11) * (1.0 / 9007199254740992.0)) - 0.5;
  }
}

// per-CTA max |x| and its index
__global__ void k_absmax(const double* __restrict__ re, const double* __restrict__ im, int64_t n,
                         double* __restrict__ pval, int64_t* __restrict__ pidx) {
  __shared__ double sv[RED_THREADS];
  __shared__ int64_t si[RED_THREADS];
  double best = -1.0;
  int64_t bi = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double a = re[i] * re[i] + im[i] * im[i];
    if (a > best) { best = a; bi = i; }
  }
  sv[threadIdx.x] = best;
  si[threadIdx.x] = bi;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      double o = sv[threadIdx.x + s];
      int64_t oi = si[threadIdx.x + s];
      if (o > sv[threadIdx.x] || (o == sv[threadIdx.x] && oi < si[threadIdx.x])) {
        sv[threadIdx.x] = o;
        si[threadIdx.x] = oi;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    pval[blockIdx.x] = sv[0];
    pidx[blockIdx.x] = si[0];
  }
}

// x *= phase; drop |x| <= thr; FixComplexPrecision (sparse_interface.cpp:28-32)
__global__ void k_phase_drop(double* __restrict__ re, double* __restrict__ im, int64_t n, double pr, double pi,
                             double thr) {
  const double eps = 2.220446049250313e-16;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double a = re[i], b = im[i];
    double xr = a * pr - b * pi, xi = a * pi + b * pr;
    if (sqrt(xr * xr + xi * xi) > thr) {
      if (fabs(xi / xr) < eps) xi = 0.0;
      else if (fabs(xr / xi) < eps) xr = 0.0;
    } else {
      xr = 0.0;
      xi = 0.0;
    }
    re[i] = xr;
    im[i] = xi;
  }
}

// y = sum_j c_j V_j (c real)
__global__ void k_combine(const double* __restrict__ Vr, const double* __restrict__ Vi, int64_t ldv, int k,
                          const double* __restrict__ c, double* __restrict__ yr, double* __restrict__ yi, int64_t n) {
  __shared__ double cs[128];
  for (int j = threadIdx.x; j < k; j += blockDim.x) cs[j] = c[j];
  __syncthreads();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double xr = 0.0, xi = 0.0;
    for (int j = 0; j < k; ++j) {
      xr += cs[j] * Vr[(int64_t)j * ldv + i];
      xi += cs[j] * Vi[(int64_t)j * ldv + i];
    }
    yr[i] = xr;
    yi[i] = xi;
  }
}

// ---- Krylov kernels with device-resident coefficients ----------------------
// The Lanczos loop keeps its coefficients on the device: a projection's
// coefficients are reduced into device memory and read back by the update
// kernel, so one iteration needs no host round trip.
constexpr int KR_THREADS = 256;
constexpr int KR_E = 8;  // elements per thread per tile: w is read once, into registers

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// partial[r][blk]: r = 2j, 2j+1 -> <V_j, w> (re, im) for j < k; r = 2k -> |w|^2.
// One pass over w (held in registers per tile) and one over each V_j.
// With `uc` set, w -= c u (c = uc[0] + i uc[1], u = (ur, ui)) first, written
// back, and the products are taken with the updated w.
__global__ void __launch_bounds__(KR_THREADS)
k_mdot(const double* __restrict__ Vr, const double* __restrict__ Vi, int64_t ldv, int k, double* __restrict__ wr,
       double* __restrict__ wi, int64_t n, const double* __restrict__ uc, const double* __restrict__ ur,
       const double* __restrict__ ui, double* __restrict__ partial) {
  extern __shared__ double acc[];  // [warps][2k + 1], one row per warp: no shared-memory atomics
  const int nw = KR_THREADS / 32, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int rows = 2 * k + 1;
  for (int t = threadIdx.x; t < nw * rows; t += blockDim.x) acc[t] = 0.0;
  __syncthreads();
  const int64_t tile = (int64_t)KR_THREADS * KR_E;
  for (int64_t base = (int64_t)blockIdx.x * tile; base < n; base += (int64_t)gridDim.x * tile) {
    double xr[KR_E], xi[KR_E];
    double s = 0.0;
#pragma unroll
    for (int e = 0; e < KR_E; ++e) {
      const int64_t i = base + (int64_t)e * KR_THREADS + threadIdx.x;
      xr[e] = i < n ? wr[i] : 0.0;
      xi[e] = i < n ? wi[i] : 0.0;
      if (uc && i < n) {
        const double cr = uc[0], ci = uc[1], a = ur[i], b = ui[i];
        xr[e] -= cr * a - ci * b;
        xi[e] -= cr * b + ci * a;
        wr[i] = xr[e];
        wi[i] = xi[e];
      }
      s += xr[e] * xr[e] + xi[e] * xi[e];
    }
    s = warp_sum(s);
    if (lane == 0) acc[warp * rows + 2 * k] += s;
    for (int j = 0; j < k; ++j) {
      const double* vr = Vr + (int64_t)j * ldv;
      const double* vi = Vi + (int64_t)j * ldv;
      double sr = 0.0, si = 0.0;
#pragma unroll
      for (int e = 0; e < KR_E; ++e) {
        const int64_t i = base + (int64_t)e * KR_THREADS + threadIdx.x;
        if (i < n) {
          const double ar = vr[i], ai = vi[i];
          sr += ar * xr[e] + ai * xi[e];
          si += ar * xi[e] - ai * xr[e];
        }
      }
      sr = warp_sum(sr);
      si = warp_sum(si);
      if (lane == 0) {
        acc[warp * rows + 2 * j] += sr;
        acc[warp * rows + 2 * j + 1] += si;
      }
    }
  }
  __syncthreads();
  for (int r = threadIdx.x; r < rows; r += blockDim.x) {
    double t = 0.0;
    for (int w = 0; w < nw; ++w) t += acc[w * rows + r];
    partial[(int64_t)r * gridDim.x + blockIdx.x] = t;
  }
}

// w -= sum_j h_j V_j (h complex, on the device); partial[blk] = |w|^2 over
// this CTA's elements afterwards.
__global__ void __launch_bounds__(KR_THREADS)
k_maxpy_norm(const double* __restrict__ Vr, const double* __restrict__ Vi, int64_t ldv, int k,
             const double* __restrict__ h, double* __restrict__ wr, double* __restrict__ wi, int64_t n,
             double* __restrict__ partial) {
  __shared__ double hs[2 * 128];
  __shared__ double red[KR_THREADS / 32];
  for (int j = threadIdx.x; j < 2 * k; j += blockDim.x) hs[j] = h[j];
  __syncthreads();
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double xr = wr[i], xi = wi[i];
#pragma unroll 4
    for (int j = 0; j < k; ++j) {
      const double hr = hs[2 * j], hi = hs[2 * j + 1];
      const double vr = Vr[(int64_t)j * ldv + i], vi = Vi[(int64_t)j * ldv + i];
      xr -= hr * vr - hi * vi;
      xi -= hr * vi + hi * vr;
    }
    wr[i] = xr;
    wi[i] = xi;
    s += xr * xr + xi * xi;
  }
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < KR_THREADS / 32; ++w) t += red[w];
    partial[blockIdx.x] = t;
  }
}

// Local Lanczos step: w -= beta v_prev (beta = *pb, skipped when v_prev is
// null), then partial[0|1][blk] = <v, w> (re | im) over this CTA's elements.
__global__ void __launch_bounds__(KR_THREADS)
k_axpy_dot(const double* __restrict__ pr, const double* __restrict__ pi, const double* __restrict__ pb,
           const double* __restrict__ vr, const double* __restrict__ vi, double* __restrict__ wr,
           double* __restrict__ wi, int64_t n, double* __restrict__ partial) {
  __shared__ double red[2][KR_THREADS / 32];
  const double b = pr ? *pb : 0.0;
  double sr = 0.0, si = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double xr = wr[i], xi = wi[i];
    if (pr) {
      xr -= b * pr[i];
      xi -= b * pi[i];
      wr[i] = xr;
      wi[i] = xi;
    }
    const double ar = vr[i], ai = vi[i];
    sr += ar * xr + ai * xi;
    si += ar * xi - ai * xr;
  }
  sr = warp_sum(sr);
  si = warp_sum(si);
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = sr;
    red[1][threadIdx.x >> 5] = si;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    double t = 0.0;
    for (int w = 0; w < KR_THREADS / 32; ++w) t += red[threadIdx.x][w];
    partial[(int64_t)threadIdx.x * gridDim.x + blockIdx.x] = t;
  }
}

// Lanczos coefficients of step j: alpha_j = *a1 + *a2 (the real parts of the
// two projections on v_j), beta_j = |w|; scale = 1 / beta_j, or 0 when the
// Krylov space is exhausted (the next basis vector is then zero).
__global__ void k_lanczos_coef(const double* __restrict__ a1, const double* __restrict__ a2,
                               const double* __restrict__ nrm2, int j, double* __restrict__ alpha,
                               double* __restrict__ beta, double* __restrict__ scale) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double a = *a1 + *a2;
  const double b = sqrt(fmax(0.0, *nrm2));
  alpha[j] = a;
  beta[j] = b;
  *scale = b > 1e-14 * fmax(1.0, fabs(a)) ? 1.0 / b : 0.0;
}

// y = s * x with s read from the device; `inv_sqrt` takes s = 1 / sqrt(*p)
// (0 when *p is not positive).
__global__ void k_scale_dev(const double* __restrict__ xr, const double* __restrict__ xi,
                            const double* __restrict__ p, int inv_sqrt, double* __restrict__ yr,
                            double* __restrict__ yi, int64_t n) {
  const double v = *p;
  const double s = inv_sqrt ? (v > 0.0 ? 1.0 / sqrt(v) : 0.0) : v;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    yr[i] = s * xr[i];
    yi[i] = s * xi[i];
  }
}

}  // namespace

int launch_block_axpy(const AxpyBlock* d_blocks, int nblocks, const AxpyTerm* d_terms, const Planar& src,
                      Planar& dst, cudaStream_t st, bool accumulate) {
  if (nblocks == 0) return CMPS_OK;
  k_block_axpy<<<nblocks, 256, 0, st>>>(d_blocks, d_terms, src.re(), src.im(), dst.re(), dst.im(), accumulate ? 1 : 0);
  CMPS_CUDA(cudaGetLastError());
  return CMPS_OK;
}

// ---- Krylov helpers ---------------------------------------------------------
int VecOps::init(int64_t n_) {
  n = n_;
  nb = grid_for(n, RED_THREADS);
  if (nb > 1024) nb = 1024;
  CMPS_CUDA(dmalloc(&d_partial, sizeof(double) * (2 * 128 + 2) * nb));
  CMPS_CUDA(dmalloc(&d_coef, sizeof(double) * kCoefDoubles));
  CMPS_CUDA(dmalloc(&d_small, sizeof(double) * 2 * 128 * 2));
  CMPS_CUDA(dmalloc(&d_pidx, sizeof(int64_t) * nb));
  return CMPS_OK;
}

void VecOps::release() {
  if (d_partial) dfree(d_partial);
  if (d_small) dfree(d_small);
  if (d_pidx) dfree(d_pidx);
  if (d_coef) dfree(d_coef);
  d_partial = d_small = d_coef = nullptr;
  d_pidx = nullptr;
}

int VecOps::multidot(const double* Vr, const double* Vi, int64_t ldv, int k, const double* wr, const double* wi,
                     double* h_host, cudaStream_t st) {
  if (k > 128) return fail(CMPS_ERR_ARG, "krylov dimension above 128");
  k_multidot<<<nb, RED_THREADS, 2 * RED_THREADS * sizeof(double), st>>>(Vr, Vi, ldv, k, wr, wi, n, d_partial);
  CMPS_CUDA(cudaGetLastError());
  k_reduce_rows<<<2 * k, RED_THREADS, 0, st>>>(d_partial, nb, 2 * k, d_small);
  CMPS_CUDA(cudaGetLastError());
  if (h_host) {
    CMPS_CUDA(cudaMemcpyAsync(h_host, d_small, sizeof(double) * 2 * k, cudaMemcpyDeviceToHost, st));
    CMPS_CUDA(cudaStreamSynchronize(st));
  }
  return CMPS_OK;
}

int VecOps::multiaxpy(const double* Vr, const double* Vi, int64_t ldv, int k, const double* h_host, double* wr,
                      double* wi, double sign, cudaStream_t st) {
  if (k > 128) return fail(CMPS_ERR_ARG, "krylov dimension above 128");
  CMPS_CUDA(cudaMemcpyAsync(d_small + 256, h_host, sizeof(double) * 2 * k, cudaMemcpyHostToDevice, st));
  k_multiaxpy<<<grid_for(n, 256), 256, 0, st>>>(Vr, Vi, ldv, k, d_small + 256, wr, wi, n, sign);
  CMPS_CUDA(cudaGetLastError());
  return CMPS_OK;
}

int VecOps::norm2(const double* xr, const double* xi, double* out, cudaStream_t st) {
  double h[2];
  CMPS_TRY(multidot(xr, xi, 0, 1, xr, xi, h, st));
  *out = h[0];
  return CMPS_OK;
}

int VecOps::scale_copy(const double* xr, const double* xi, double s, double* yr, double* yi, cudaStream_t st) {
  k_scale_copy<<<grid_for(n, 256), 256, 0, st>>>(xr, xi, s, yr, yi, n);
  CMPS_CUDA(cudaGetLastError());
  return CMPS_OK;
}

int VecOps::random(double* re, double* im, uint64_t seed, cudaStream_t st) {
  k_random<<<grid_for(n, 256), 256, 0, st>>>(re, im, n, seed);
  CMPS_CUDA(cudaGetLastError());
  return CMPS_OK;
}

int VecOps::combine(const double* Vr, const double* Vi, int64_t ldv, int k, const double* c_host, double* yr,
                    double* yi, cudaStream_t st) {
  if (k > 128) return fail(CMPS_ERR_ARG, "krylov dimension above 128");
  CMPS_CUDA(cudaMemcpyAsync(d_small + 256, c_host, sizeof(double) * k, cudaMemcpyHostToDevice, st));
  k_combine<<<grid_for(n, 256), 256, 0, st>>>(Vr, Vi, ldv, k, d_small + 256, yr, yi, n);
  CMPS_CUDA(cudaGetLastError());
  return CMPS_OK;
}

int VecOps::absmax(const double* re, const double* im, double* val, int64_t* idx, cudaStream_t st) {
  k_absmax<<<nb, RED_THREADS, 0, st>>>(re, im, n, d_partial, d_pidx);
  CMPS_CUDA(cudaGetLastError());
  std::vector<double> pv(nb);
  std::vector<int64_t> pi(nb);
  CMPS_CUDA(cudaMemcpyAsync(pv.data(), d_partial, sizeof(double) * nb, cudaMemcpyDeviceToHost, st));
  CMPS_CUDA(cudaMemcpyAsync(pi.data(), d_pidx, sizeof(int64_t) * nb, cudaMemcpyDeviceToHost, st));
  CMPS_CUDA(cudaStreamSynchronize(st));
  double best = -1.0;
  int64_t bi = 0;
  for (int b = 0; b < nb; ++b)
    if (pv[b] > best || (pv[b] == best && pi[b] < bi)) {
      best = pv[b];
      bi = pi[b];
    }
  *val = best;
  *idx = bi;
  return CMPS_OK;
}

int VecOps::phase_drop(double* re, double* im, double pr, double pi, double thr, cudaStream_t st) {
  k_phase_drop<<<grid_for(n, 256), 256, 0, st>>>(re, im, n, pr, pi, thr);
  CMPS_CUDA(cudaGetLastError());
  return CMPS_OK;
}

int VecOps::mdot_dev(const double* Vr, const double* Vi, int64_t ldv, int k, const double* wr, const double* wi,
                     double* d_out, cudaStream_t st) {
  if (k < 0 || k > 128) return fail(CMPS_ERR_ARG, "krylov dimension above 128");
  const int64_t tile = (int64_t)KR_THREADS * KR_E;
  const int g = (int)std::max<int64_t>(1, std::min<int64_t>(nb, (n + tile - 1) / tile));
  const int rows = 2 * k + 1;
  const size_t smem = sizeof(double) * (KR_THREADS / 32) * rows;
  k_mdot<<<g, KR_THREADS, smem, st>>>(Vr, Vi, ldv, k, const_cast<double*>(wr), const_cast<double*>(wi), n, nullptr,
                                      nullptr, nullptr, d_partial);
  CMPS_CUDA(cudaGetLastError());
  k_reduce_rows<<<rows, RED_THREADS, 0, st>>>(d_partial, g, rows, d_out);
  CMPS_CUDA(cudaGetLastError());
  return CMPS_OK;
}

int VecOps::update_mdot_dev(const double* d_c, const double* ur, const double* ui, const double* Vr, const double* Vi,
                            int64_t ldv, int k, double* wr, double* wi, double* d_out, cudaStream_t st) {
  if (k < 0 || k > 128) return fail(CMPS_ERR_ARG, "krylov dimension above 128");
  const int64_t tile = (int64_t)KR_THREADS * KR_E;
  const int g = (int)std::max<int64_t>(1, std::min<int64_t>(nb, (n + tile - 1) / tile));
  const int rows = 2 * k + 1;
  const size_t smem = sizeof(double) * (KR_THREADS / 32) * rows;
  k_mdot<<<g, KR_THREADS, smem, st>>>(Vr, Vi, ldv, k, wr, wi, n, d_c, ur, ui, d_partial);
  CMPS_CUDA(cudaGetLastError());
  k_reduce_rows<<<rows, RED_THREADS, 0, st>>>(d_partial, g, rows, d_out);
  CMPS_CUDA(cudaGetLastError());
  return CMPS_OK;
}

int VecOps::axpy_dot_dev(const double* pr, const double* pi, const double* d_beta, const double* vr, const double* vi,
                         double* wr, double* wi, double* d_out, cudaStream_t st) {
  const int g = std::min(nb, grid_for(n, KR_THREADS));
  k_axpy_dot<<<g, KR_THREADS, 0, st>>>(pr, pi, d_beta, vr, vi, wr, wi, n, d_partial);
  CMPS_CUDA(cudaGetLastError());
  k_reduce_rows<<<2, RED_THREADS, 0, st>>>(d_partial, g, 2, d_out);
  CMPS_CUDA(cudaGetLastError());
  return CMPS_OK;
}

int VecOps::maxpy_norm_dev(const double* Vr, const double* Vi, int64_t ldv, int k, const double* d_h, double* wr,
                           double* wi, double* d_nrm2, cudaStream_t st) {
  if (k < 0 || k > 128) return fail(CMPS_ERR_ARG, "krylov dimension above 128");
  const int g = std::min(nb, grid_for(n, KR_THREADS));
  k_maxpy_norm<<<g, KR_THREADS, 0, st>>>(Vr, Vi, ldv, k, d_h, wr, wi, n, d_partial);
  CMPS_CUDA(cudaGetLastError());
  k_reduce_rows<<<1, RED_THREADS, 0, st>>>(d_partial, g, 1, d_nrm2);
  CMPS_CUDA(cudaGetLastError());
  return CMPS_OK;
}

int VecOps::lanczos_coef(const double* d_a1, const double* d_a2, const double* d_nrm2, int j, double* d_alpha,
                         double* d_beta, double* d_scale, cudaStream_t st) {
  k_lanczos_coef<<<1, 32, 0, st>>>(d_a1, d_a2, d_nrm2, j, d_alpha, d_beta, d_scale);
  CMPS_CUDA(cudaGetLastError());
  return CMPS_OK;
}

int VecOps::scale_dev(const double* xr, const double* xi, const double* d_s, bool inv_sqrt, double* yr, double* yi,
                      cudaStream_t st) {
  k_scale_dev<<<grid_for(n, 256), 256, 0, st>>>(xr, xi, d_s, inv_sqrt ? 1 : 0, yr, yi, n);
  CMPS_CUDA(cudaGetLastError());
  return CMPS_OK;
}

}  // namespace cmps
