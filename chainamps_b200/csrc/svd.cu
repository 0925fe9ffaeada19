// Charge-block SVD truncation of the two-vertex wavefunction and the
// environment updates that consume its factors.
//
// SVD (SparseMatrix::SVD, sparse_interface.cpp:1248-1406): for every
// middle-charge block Theta_m (the column-charge blocks of
// GetAllBlockColumns, MPX_matrix.cpp:365-385): skip it if its weight is
// <= eps^2; restrict to its non-empty rows and columns (TranslationBlock,
// sparse_interface.hpp:367-376); FP64 SVD on the device (cuSOLVER gesvdj);
// drop |u| <= eps/rows and |v| <= eps/cols.  Then the global descending
// sort (ties: first seen), chi cap, truncation-weight cut and 1e-3
// degeneracy extension decide the kept count of every block.
//
// Environment updates (MakeLeftBlock / MakeRightBlock,
// DMRG_routines.cpp:594-611) reuse the handle's LeftPart / RightPart:
//   L'^{b1} = U^H (LeftPart^{b1} U),   R'^{b1} = (V^dag RightPart^{b1}) V^dag^H
// as grouped GEMMs; the blocks stay on the device.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <atomic>
#include <thread>
#include <set>

#include "heff.h"

namespace cmps {

static const double kEps = 2.220446049250313e-16;

// Worker streams and handles for factoring the SVD's sectors concurrently:
// cuSOLVER's dense eigensolver runs one sector far below the GPU's capacity,
// so independent sectors run side by side, one host thread per worker.
struct SvdWorker {
  cudaStream_t st = nullptr;
  cusolverDnHandle_t sol = nullptr;
  cublasHandle_t blas = nullptr;
};
struct SvdPool {
  std::vector<SvdWorker> w;
};
constexpr int kSvdWorkers = 6;

static int get_pool(cmps_context* ctx, SvdPool** out) {
  if (!ctx->svd_pool) {
    auto* p = new SvdPool();
    ctx->svd_pool = p;
    p->w.resize(kSvdWorkers);
    for (SvdWorker& w : p->w) {
      if (cudaStreamCreateWithFlags(&w.st, cudaStreamNonBlocking) != cudaSuccess)
        return fail(CMPS_ERR_CUDA, "SVD worker stream creation failed");
      if (cusolverDnCreate(&w.sol) != CUSOLVER_STATUS_SUCCESS) return fail(CMPS_ERR_CUDA, "cusolverDnCreate failed");
      if (cublasCreate(&w.blas) != CUBLAS_STATUS_SUCCESS) return fail(CMPS_ERR_CUDA, "cublasCreate failed");
      cusolverDnSetStream(w.sol, w.st);
      cublasSetStream(w.blas, w.st);
    }
    // first use of a handle loads and sets up its kernels: do it here, once,
    // with a 2 x 2 eigenproblem and GEMM per worker, not inside a step's SVD
    cuDoubleComplex* a = nullptr;
    double* wv = nullptr;
    int* info = nullptr;
    if (dmalloc(&a, sizeof(cuDoubleComplex) * 8) == cudaSuccess && dmalloc(&wv, sizeof(double) * 2) == cudaSuccess &&
        dmalloc(&info, sizeof(int)) == cudaSuccess) {
      const cuDoubleComplex id[4] = {{1, 0}, {0, 0}, {0, 0}, {1, 0}};
      for (SvdWorker& w : p->w) {
        cudaMemcpyAsync(a, id, sizeof(id), cudaMemcpyHostToDevice, w.st);
        int lw = 0;
        cusolverDnZheevd_bufferSize(w.sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, 2, a, 2, wv, &lw);
        cuDoubleComplex* work = nullptr;
        if (dmalloc(&work, sizeof(cuDoubleComplex) * std::max(1, lw)) == cudaSuccess) {
          cusolverDnZheevd(w.sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, 2, a, 2, wv, work, lw, info);
          const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
          cublasZgemm(w.blas, CUBLAS_OP_N, CUBLAS_OP_C, 2, 2, 2, &one, a, 2, a, 2, &zero, a + 4, 2);
          cudaStreamSynchronize(w.st);
          dfree(work);
        }
      }
    }
    if (a) dfree(a);
    if (wv) dfree(wv);
    if (info) dfree(info);
  }
  *out = (SvdPool*)ctx->svd_pool;
  return CMPS_OK;
}

void release_solver(cmps_context* ctx) {
  if (ctx && ctx->svd_pool) {
    auto* p = (SvdPool*)ctx->svd_pool;
    for (SvdWorker& w : p->w) {
      if (w.sol) cusolverDnDestroy(w.sol);
      if (w.blas) cublasDestroy(w.blas);
      if (w.st) cudaStreamDestroy(w.st);
    }
    delete p;
    ctx->svd_pool = nullptr;
  }
  if (ctx && ctx->solver) {
    cusolverDnDestroy((cusolverDnHandle_t)ctx->solver);
    ctx->solver = nullptr;
  }
  if (ctx && ctx->blas) {
    cublasDestroy((cublasHandle_t)ctx->blas);
    ctx->blas = nullptr;
  }
}

static int get_blas(cmps_context* ctx, cublasHandle_t* out) {
  if (!ctx->blas) {
    cublasHandle_t h;
    if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) return fail(CMPS_ERR_CUDA, "cublasCreate failed");
    ctx->blas = h;
  }
  cublasSetStream((cublasHandle_t)ctx->blas, ctx->stream);
  *out = (cublasHandle_t)ctx->blas;
  return CMPS_OK;
}

static int get_solver(cmps_context* ctx, cusolverDnHandle_t* out) {
  if (!ctx->solver) {
    cusolverDnHandle_t h;
    if (cusolverDnCreate(&h) != CUSOLVER_STATUS_SUCCESS) return fail(CMPS_ERR_CUDA, "cusolverDnCreate failed");
    ctx->solver = h;
  }
  cusolverDnSetStream((cusolverDnHandle_t)ctx->solver, ctx->stream);
  *out = (cusolverDnHandle_t)ctx->solver;
  return CMPS_OK;
}

int context_blas(cmps_context* ctx, void** out) {
  cublasHandle_t h;
  CMPS_TRY(get_blas(ctx, &h));
  *out = h;
  return CMPS_OK;
}

int context_solver(cmps_context* ctx, void** out) {
  cusolverDnHandle_t h;
  CMPS_TRY(get_solver(ctx, &h));
  *out = h;
  return CMPS_OK;
}

namespace {

__global__ void k_nzflags(const double* __restrict__ re, const double* __restrict__ im, int64_t rows,
                          int64_t cols, int* __restrict__ rflag, int* __restrict__ cflag,
                          double* __restrict__ weight) {
  double w = 0.0;
  int64_t n = rows * cols;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    double a = re[e], b = im[e];
    if (a != 0.0 || b != 0.0) {
      rflag[e / cols] = 1;
      cflag[e % cols] = 1;
      w += a * a + b * b;
    }
  }
  for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
  if ((threadIdx.x & 31) == 0 && w != 0.0) atomicAdd(weight, w);
}

// compacted block, column-major interleaved: A[i + nr*j] = Theta[rows[i], cols[j]]
__global__ void k_gather_cm(const double* __restrict__ re, const double* __restrict__ im, int64_t ld,
                            const int64_t* __restrict__ rows, int64_t nr, const int64_t* __restrict__ cols,
                            int64_t nc, double2* __restrict__ A) {
  int64_t n = nr * nc;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    int64_t i = e % nr, j = e / nr;
    int64_t o = rows[i] * ld + cols[j];
    A[e] = make_double2(re[o], im[o]);
  }
}

// U_m[rows[i], j] = Ucm[i + nr*j] (j < k), |u| <= thr dropped; U_m row-major ld = k.
__global__ void k_scatter_u(const double2* __restrict__ Ucm, int64_t nr, int64_t k, const int64_t* __restrict__ rows,
                            double thr, double* __restrict__ ur, double* __restrict__ ui) {
  int64_t n = nr * k;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    int64_t i = e % nr, j = e / nr;
    double2 v = Ucm[e];
    bool keep = sqrt(v.x * v.x + v.y * v.y) > thr;
    int64_t o = rows[i] * k + j;
    ur[o] = keep ? v.x : 0.0;
    ui[o] = keep ? v.y : 0.0;
  }
}

// Vd_m[j, cols[c]] = conj(Vcm[c + nc*j]); Vd_m row-major ld = ncols.
__global__ void k_scatter_vd(const double2* __restrict__ Vcm, int64_t nc, int64_t k, const int64_t* __restrict__ cols,
                             int64_t ld, double thr, double* __restrict__ vr, double* __restrict__ vi) {
  int64_t n = nc * k;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    int64_t c = e % nc, j = e / nc;
    double2 v = Vcm[e];
    bool keep = sqrt(v.x * v.x + v.y * v.y) > thr;
    int64_t o = j * ld + cols[c];
    vr[o] = keep ? v.x : 0.0;
    vi[o] = keep ? -v.y : 0.0;
  }
}

// F[:, j] = E[:, p-1-j] (eigenvectors in descending eigenvalue order)
__global__ void k_reverse_cols(const double2* __restrict__ E, int64_t p, double2* __restrict__ F) {
  const int64_t n = p * p;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e % p, j = e / p;
    F[e] = E[i + p * (p - 1 - j)];
  }
}

// X[e] = two uniform values in [-1, 1) from a counter hash (splitmix64) of
// (seed, e): the Gaussian-free test matrix of the range finder.
__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
__global__ void k_fill_random(double2* __restrict__ X, int64_t n, uint64_t seed) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t h = splitmix64(seed ^ splitmix64((uint64_t)e));
    const double a = (double)(h >> 32) * (1.0 / 4294967296.0), b = (double)(h & 0xffffffffull) * (1.0 / 4294967296.0);
    X[e] = make_double2(2.0 * a - 1.0, 2.0 * b - 1.0);
  }
}

// out[j] = |R[:, j] - s[j] F[:, j]|^2 (column-major rows x cols, one block per column)
__global__ void __launch_bounds__(256) k_col_resid(const double2* __restrict__ R, const double2* __restrict__ F,
                                                   const double* __restrict__ s, int64_t rows,
                                                   double* __restrict__ out) {
  __shared__ double part[8];
  const int64_t j = blockIdx.x;
  const double sj = s[j];
  double acc = 0.0;
  for (int64_t i = threadIdx.x; i < rows; i += blockDim.x) {
    const double2 r = R[i + rows * j], f = F[i + rows * j];
    const double x = r.x - sj * f.x, y = r.y - sj * f.y;
    acc += x * x + y * y;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += part[w];
    out[j] = t;
  }
}

// G[i][i] += c * trace(G) (one block): the shift of shifted Cholesky QR,
// with the Frobenius norm squared (the trace of the Gram matrix) standing in
// for the squared 2-norm.
__global__ void __launch_bounds__(256) k_shift_diag(double2* __restrict__ G, int64_t n, double c) {
  __shared__ double part[8];
  __shared__ double tr;
  double acc = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) acc += G[i + n * i].x;
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += part[w];
    tr = t;
  }
  __syncthreads();
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) G[i + n * i].x += c * tr;
}

// flag |= (info != 0): a Cholesky factorisation that broke down
__global__ void k_or_info(const int* __restrict__ info, int* __restrict__ flag) {
  if (threadIdx.x == 0 && blockIdx.x == 0 && *info != 0) *flag = 1;
}

// Sum of |X[e]|^2 in a fixed order: kSumBlocks partial sums, then one block
// adds them (no atomics, so the result does not depend on scheduling).
constexpr int kSumBlocks = 512;
__global__ void __launch_bounds__(256) k_sumsq_partial(const double2* __restrict__ X, int64_t n,
                                                       double* __restrict__ part) {
  __shared__ double wsum[8];
  double acc = 0.0;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const double2 v = X[e];
    acc += v.x * v.x + v.y * v.y;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += wsum[w];
    part[blockIdx.x] = t;
  }
}
__global__ void k_sum_final(const double* __restrict__ part, int n, double* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < n; ++i) t += part[i];
    *out = t;
  }
}

// G[:, j] /= s[j]  (column-major, rows x cols); zero columns where s[j] == 0
// G (b x b, column-major) = R^H for the upper triangle R of a Householder QR
// held in Z (column-major, leading dimension ld).
__global__ void k_upper_adjoint(const double2* __restrict__ Z, int64_t ld, int64_t b, double2* __restrict__ G) {
  const int64_t n = b * b;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e % b, j = e / b;
    double2 v = make_double2(0.0, 0.0);
    if (j <= i) {
      const double2 r = Z[j + i * ld];  // R(j, i)
      v = make_double2(r.x, -r.y);
    }
    G[e] = v;
  }
}

__global__ void k_scale_cols_inv(double2* __restrict__ G, int64_t rows, int64_t cols, const double* __restrict__ s) {
  const int64_t n = rows * cols;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = e / rows;
    const double f = s[j] > 0.0 ? 1.0 / s[j] : 0.0;
    G[e].x *= f;
    G[e].y *= f;
  }
}

// M[r + R c] = rs[r] cs[c] Vd[src[r] + c]  (column-major gather of
// Lambda V^dagger diag(prev_lambda) restricted to one a2 sector)
__global__ void k_gather_fid(const double* __restrict__ vr, const double* __restrict__ vi,
                             const int64_t* __restrict__ src, const double* __restrict__ rs,
                             const double* __restrict__ cs, int64_t R, int64_t Cn, double2* __restrict__ M) {
  const int64_t n = R * Cn;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e % R, c = e / R;
    const double f = rs[r] * cs[c];
    M[e] = make_double2(f * vr[src[r] + c], f * vi[src[r] + c]);
  }
}

int grid_of(int64_t n) {
  int64_t g = (n + 255) / 256;
  if (g < 1) g = 1;
  if (g > 148 * 16) g = 148 * 16;
  return (int)g;
}

}  // namespace

// Kept count of SparseMatrix::SVD (sparse_interface.cpp:1346-1376).
static int64_t truncation_length(const std::vector<double>& sv, int64_t D, double max_trunc,
                                 bool* weight_decided = nullptr) {
  const int64_t N = (int64_t)sv.size();
  int64_t length = (D > 0 && D < N) ? D : N;
  const int64_t cap = length;
  double trunc_error = 0.0;
  int64_t tl = N;
  while (trunc_error < max_trunc && tl > 0) {
    trunc_error += sv[tl - 1] * sv[tl - 1];
    --tl;
  }
  ++tl;
  if (tl < length) length = tl;
  if (weight_decided) *weight_decided = tl < cap;
  while (length < N && (sv[length - 1] - sv[length]) / sv[length - 1] < 1.0e-3) ++length;
  return length;
}

int theta_svd(Heff& H, int64_t chi, double max_trunc, SvdResult& out, const std::map<QKey, int64_t>* kept_hint) {
  if (!H.have_theta) return fail(CMPS_ERR_STATE, "no wavefunction: call cmps_heff_eigs or cmps_heff_set_theta first");
  cudaStream_t st = H.ctx->stream;
  cusolverDnHandle_t sol;
  CMPS_TRY(get_solver(H.ctx, &sol));
  const ThetaSpace& th = H.th;
  const int nm = (int)th.mq.size();
  out.rules = H.rules;
  out.d = H.d;
  out.sigq = H.sigq;
  out.a0 = H.L.a;
  out.a2 = H.R.a;
  out.th = th;
  struct Blk {
    std::vector<int64_t> rows, cols;
    std::vector<double> s;
    bool eig = false;
    // randomized route: only the leading s.size() triplets were computed;
    // tail = |A - Q Q^H A|_F^2 (the weight outside the range found),
    // resid[j] = |A v_j - s_j u_j| (or its transpose form)
    bool rnd = false;
    bool red_exact = false;  // the reduced b x b problem by QR + Jacobi SVD (else Hermitian eigensolver)
    double tail = 0.0;
    std::vector<double> resid;
    int64_t bb = 0;  // triplets the randomized route computed
    double2* dU = nullptr;
    double2* dV = nullptr;
    int64_t* drows = nullptr;
    int64_t* dcols = nullptr;
  };
  std::vector<Blk> blk(nm);
  int64_t maxr = 1, maxc = 1;
  for (int m = 0; m < nm; ++m) {
    maxr = std::max(maxr, th.nrows[m]);
    maxc = std::max(maxc, th.ncols[m]);
  }
  int* dflags = nullptr;
  double* dweight = nullptr;
  double2* dA = nullptr;
  double* dS = nullptr;
  int* dinfo = nullptr;
  auto cleanup = [&]() {
    if (dflags) dfree(dflags);
    if (dweight) dfree(dweight);
    if (dA) dfree(dA);
    if (dS) dfree(dS);
    if (dinfo) dfree(dinfo);
    for (auto& b : blk) {
      if (b.dU) dfree(b.dU);
      if (b.dV) dfree(b.dV);
      if (b.drows) dfree(b.drows);
      if (b.dcols) dfree(b.dcols);
    }
  };
  int status = CMPS_OK;
  do {
    if (dmalloc(&dflags, sizeof(int) * (maxr + maxc)) != cudaSuccess ||
        dmalloc(&dweight, sizeof(double)) != cudaSuccess ||
        dmalloc(&dA, sizeof(double2) * maxr * maxc) != cudaSuccess ||
        dmalloc(&dS, sizeof(double) * std::min(maxr, maxc)) != cudaSuccess ||
        dmalloc(&dinfo, sizeof(int)) != cudaSuccess) {
      status = fail(CMPS_ERR_NOMEM, "SVD workspace allocation failed");
      break;
    }
    gesvdjInfo_t params;
    cusolverDnCreateGesvdjInfo(&params);
    cusolverDnXgesvdjSetTolerance(params, 0.0);   // 0: machine precision
    cusolverDnXgesvdjSetMaxSweeps(params, 100);
    cusolverDnXgesvdjSetSortEig(params, 1);
    cublasHandle_t blas;
    if ((status = get_blas(H.ctx, &blas)) != CMPS_OK) break;
    // ---- pass 1: empty-block skip and row/column pruning ----
    for (int m = 0; m < nm && status == CMPS_OK; ++m) {
      const int64_t R = th.nrows[m], C = th.ncols[m];
      if (R == 0 || C == 0) continue;
      const double* bre = H.theta.re() + th.base[m];
      const double* bim = H.theta.im() + th.base[m];
      cudaMemsetAsync(dflags, 0, sizeof(int) * (R + C), st);
      cudaMemsetAsync(dweight, 0, sizeof(double), st);
      k_nzflags<<<grid_of(R * C), 256, 0, st>>>(bre, bim, R, C, dflags, dflags + R, dweight);
      std::vector<int> fl(R + C);
      double w = 0.0;
      cudaMemcpyAsync(fl.data(), dflags, sizeof(int) * (R + C), cudaMemcpyDeviceToHost, st);
      cudaMemcpyAsync(&w, dweight, sizeof(double), cudaMemcpyDeviceToHost, st);
      if (cudaStreamSynchronize(st) != cudaSuccess) { status = fail(CMPS_ERR_CUDA, "SVD flag pass failed"); break; }
      if (w <= kEps * kEps) continue;  // empty block (sparse_interface.cpp:1279)
      Blk& b = blk[m];
      for (int64_t i = 0; i < R; ++i) if (fl[i]) b.rows.push_back(i);
      for (int64_t j = 0; j < C; ++j) if (fl[R + j]) b.cols.push_back(j);
      const int64_t nr = (int64_t)b.rows.size(), nc = (int64_t)b.cols.size();
      const int64_t mn = std::min(nr, nc);
      if (dmalloc(&b.drows, sizeof(int64_t) * nr) != cudaSuccess ||
          dmalloc(&b.dcols, sizeof(int64_t) * nc) != cudaSuccess ||
          dmalloc(&b.dU, sizeof(double2) * nr * mn) != cudaSuccess ||
          dmalloc(&b.dV, sizeof(double2) * nc * mn) != cudaSuccess) {
        status = fail(CMPS_ERR_NOMEM, "SVD block allocation failed");
        break;
      }
      cudaMemcpyAsync(b.drows, b.rows.data(), sizeof(int64_t) * nr, cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(b.dcols, b.cols.data(), sizeof(int64_t) * nc, cudaMemcpyHostToDevice, st);
    }
    if (status != CMPS_OK) { cusolverDnDestroyGesvdjInfo(params); break; }
    // ---- pass 2: factor every block ----
    // exact: one-sided Jacobi SVD (gesvdj).  Otherwise, for sectors of at least
    // kEigMin rows and columns, the Hermitian route: eigenpairs of the smaller
    // Gram matrix (A A^H or A^H A, zheevd), the other factor by one GEMM.  Its
    // singular values carry an absolute error ~eps * s_max, so it is only
    // accepted below when the bond-dimension cap, not the weight cut, decides
    // the kept count and every kept value is far above that floor.
    const int64_t kEigMin = 192;
    // Streams, handles and workspaces of one factoring thread.  Buffers with
    // capacity 0 are allocated per sector (the sequential path); the
    // concurrent workers get them sized up front, so that no allocation (and
    // no device-wide synchronisation of a free) happens while they run.
    struct FW {
      cudaStream_t st;
      cusolverDnHandle_t sol;
      cublasHandle_t blas;
      gesvdjInfo_t params;
      double2* dA;
      double* dS;
      int* dinfo;
      double2* G = nullptr;
      size_t Gcap = 0;
      double2* X = nullptr;  // scratch of the randomized route
      size_t Xcap = 0;
      double* W = nullptr;
      size_t Wcap = 0;
      cuDoubleComplex* work = nullptr;
      size_t workcap = 0;
    };
    // Randomized route (Halko, Martinsson and Tropp, SIAM Review 53 (2011)
    // 217, algorithms 4.4 and 5.1) for a sector much larger than the bond
    // dimension: no sector keeps more than chi values, so its leading
    // bb = chi + kRandPad triplets suffice whenever the checks of the global
    // selection pass.  Range of M (the sector, or its adjoint when it is
    // tall) by kRandIters subspace iterations with Cholesky QR
    // re-orthonormalisation from a random start; then the SVD of the small
    // matrix B = Q^H M itself: a Householder QR B^H = Q_B R and a one-sided
    // Jacobi SVD of the bb x bb matrix R^H, so small singular values keep an
    // absolute error of ~eps s_0 (the eigenvalues of B B^H would square it).
    // Besides the triplets it records every triplet's residual and the
    // weight outside the range found.
    const int64_t kRandPad = 32;
    const int kRandIters = 2;
    // With a hint -- the values the sector of the same charge kept at the
    // previous step -- the range is 2.5 times that plus 64 (at least 64),
    // not the whole chi + kRandPad: the tail check (3) widens it where the
    // spectrum needs more.
    auto rand_b = [&](int m, int64_t mn) -> int64_t {
      if (chi <= 0 || mn < kEigMin) return 0;
      int64_t bb = std::min<int64_t>(mn, chi + kRandPad);
      if (kept_hint) {
        auto it = kept_hint->find(th.mq[m]);
        if (it != kept_hint->end()) bb = std::min<int64_t>(bb, std::max<int64_t>(64, 5 * it->second / 2 + 64));
      }
      return 4 * bb <= 3 * mn ? bb : 0;
    };
    auto rand_scratch = [&](int64_t nr, int64_t nc, int64_t bb) -> size_t {
      const int64_t pp = std::min(nr, nc), ll = std::max(nr, nc);
      return (size_t)(2 * pp * bb + 2 * ll * bb + 2 * bb * bb + 2 * bb + kSumBlocks / 2 + 2);
    };
    auto rand_lwork = [&](cusolverDnHandle_t sol, gesvdjInfo_t prm, int64_t ll, int64_t bb, int* lw) -> int {
      const int b32 = (int)bb, l32 = (int)ll;
      int a = 0, q = 0, u = 0, g = 0, e = 0, q2 = 0, u2 = 0;
      cuDoubleComplex* any = (cuDoubleComplex*)dA;
      if (cusolverDnZheevd_bufferSize(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, b32, any, b32, dS, &e) !=
              CUSOLVER_STATUS_SUCCESS ||
          cusolverDnZpotrf_bufferSize(sol, CUBLAS_FILL_MODE_UPPER, b32, any, b32, &a) != CUSOLVER_STATUS_SUCCESS ||
          cusolverDnZgeqrf_bufferSize(sol, l32, b32, any, l32, &q) != CUSOLVER_STATUS_SUCCESS ||
          cusolverDnZungqr_bufferSize(sol, l32, b32, b32, any, l32, any, &u) != CUSOLVER_STATUS_SUCCESS ||
          cusolverDnZgeqrf_bufferSize(sol, b32, b32, any, b32, &q2) != CUSOLVER_STATUS_SUCCESS ||
          cusolverDnZungqr_bufferSize(sol, b32, b32, b32, any, b32, any, &u2) != CUSOLVER_STATUS_SUCCESS ||
          cusolverDnZgesvdj_bufferSize(sol, CUSOLVER_EIG_MODE_VECTOR, 1, b32, b32, any, b32, dS, any, b32, any, b32, &g,
                                       prm) != CUSOLVER_STATUS_SUCCESS)
        return fail(CMPS_ERR_SOLVER, "randomized SVD buffer query failed");
      *lw = std::max(std::max(std::max(a, q), std::max(u, g)), std::max(std::max(e, 1), std::max(q2, u2)));
      return CMPS_OK;
    };
    auto factor_rand = [&](int m, int64_t bb, FW& fw) -> int {
      const cudaStream_t st = fw.st;
      const cusolverDnHandle_t sol = fw.sol;
      const cublasHandle_t blas = fw.blas;
      double2* const dA = fw.dA;
      double* const dS = fw.dS;
      int* const dinfo = fw.dinfo;
      Blk& b = blk[m];
      const int64_t nr = (int64_t)b.rows.size(), nc = (int64_t)b.cols.size();
      const bool left = nr <= nc;  // M = A (short side rows) or M = A^H
      const int64_t pp = left ? nr : nc, ll = left ? nc : nr;
      const cublasOperation_t opM = left ? CUBLAS_OP_N : CUBLAS_OP_C, opMH = left ? CUBLAS_OP_C : CUBLAS_OP_N;
      const size_t need = rand_scratch(nr, nc, bb);
      double2* X = fw.X;
      const bool ownX = need > fw.Xcap;
      if (ownX && dmalloc(&X, sizeof(double2) * need) != cudaSuccess)
        return fail(CMPS_ERR_NOMEM, "randomized SVD scratch allocation failed");
      int lwork = 0;
      int rc = rand_lwork(sol, fw.params, ll, bb, &lwork);
      cuDoubleComplex* work = fw.work;
      const bool ownW = rc == CMPS_OK && (size_t)lwork > fw.workcap;
      if (ownW && dmalloc(&work, sizeof(cuDoubleComplex) * (size_t)lwork) != cudaSuccess)
        rc = fail(CMPS_ERR_NOMEM, "randomized SVD work allocation failed");
      double2* const Y = X;              // pp x bb: range basis Q
      double2* const Z = Y + pp * bb;    // ll x bb: test matrix, then M^H Q = B^H, then Q_B
      double2* const Z2 = Z + ll * bb;   // ll x bb: B^H kept for the tail
      double2* const R = Z2 + ll * bb;   // pp x bb: left vectors of R^H, then M O
      double2* const Gb = R + pp * bb;   // bb x bb: Gram matrices of the QR, then R^H
      double2* const Vb = Gb + bb * bb;  // bb x bb: right vectors of R^H
      double2* const tau = Vb + bb * bb; // bb: Householder scalars
      double* const W = (double*)(tau + bb);
      double* const rs = W + bb;
      double* const part = rs + bb;
      double* const tailp = part + kSumBlocks;
      int* const chol_bad = (int*)(tailp + 1);
      const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0),
                            mone = make_cuDoubleComplex(-1.0, 0.0);
      auto zg = [&](cublasOperation_t ta, cublasOperation_t tb, int64_t M_, int64_t N_, int64_t K_,
                    const cuDoubleComplex* al, const double2* A_, int64_t lda, const double2* B_, int64_t ldb,
                    const cuDoubleComplex* be, double2* C_, int64_t ldc) {
        if (rc != CMPS_OK) return;
        if (cublasZgemm(blas, ta, tb, (int)M_, (int)N_, (int)K_, al, (const cuDoubleComplex*)A_, (int)lda,
                        (const cuDoubleComplex*)B_, (int)ldb, be, (cuDoubleComplex*)C_, (int)ldc) !=
            CUBLAS_STATUS_SUCCESS)
          rc = fail(CMPS_ERR_CUDA, "randomized SVD GEMM failed");
      };
      // Orthonormal basis of the columns of A_ (rows x bb, in place): shifted
      // Cholesky QR followed by two plain passes (shifted CholeskyQR3,
      // Fukaya, Kannan, Nakatsukasa, Yamamoto and Yanagisawa, SIAM J. Sci.
      // Comput. 42 (2020) A477), stable up to a condition number ~1/eps.  A
      // Cholesky factorisation that breaks down (a sketch of a spectrum that
      // decays below eps within the range) is redone by Householder QR
      // (geqrf, ungqr) from a copy of A_ kept in Z2, which is free until B^H
      // is formed; chol_bad stays set only if that fails too, and the sector
      // then goes to the Gram route.
      bool qr_unrecovered = false;  // a breakdown the Householder redo did not repair
      auto qr = [&](double2* A_, int64_t rows) {
        if (rc != CMPS_OK) return;
        if (cudaMemcpyAsync(Z2, A_, sizeof(double2) * rows * bb, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
            cudaMemsetAsync(chol_bad, 0, sizeof(int), st) != cudaSuccess) {
          rc = fail(CMPS_ERR_CUDA, "randomized SVD: QR copy failed");
          return;
        }
        for (int pass = 0; pass < 3 && rc == CMPS_OK; ++pass) {
          zg(CUBLAS_OP_C, CUBLAS_OP_N, bb, bb, rows, &one, A_, rows, A_, rows, &zero, Gb, bb);
          if (rc != CMPS_OK) return;
          if (pass == 0)
            k_shift_diag<<<1, 256, 0, st>>>(Gb, bb, 11.0 * ((double)rows * bb + (double)bb * (bb + 1)) * kEps);
          if (cusolverDnZpotrf(sol, CUBLAS_FILL_MODE_UPPER, (int)bb, (cuDoubleComplex*)Gb, (int)bb, work, lwork,
                               dinfo) != CUSOLVER_STATUS_SUCCESS) {
            rc = fail(CMPS_ERR_SOLVER, "randomized SVD Cholesky failed");
            return;
          }
          k_or_info<<<1, 32, 0, st>>>(dinfo, chol_bad);
          if (cublasZtrsm(blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, (int)rows,
                          (int)bb, &one, (const cuDoubleComplex*)Gb, (int)bb, (cuDoubleComplex*)A_, (int)rows) !=
              CUBLAS_STATUS_SUCCESS)
            rc = fail(CMPS_ERR_CUDA, "randomized SVD triangular solve failed");
        }
        if (rc != CMPS_OK) return;
        int broke = 0;
        if (cudaMemcpyAsync(&broke, chol_bad, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
          rc = fail(CMPS_ERR_CUDA, "randomized SVD: QR check failed");
          return;
        }
        if (!broke) return;
        // Householder QR of the kept copy: A_ = Q R, Q (rows x bb) into A_
        int hinfo = 0;
        if (cudaMemcpyAsync(A_, Z2, sizeof(double2) * rows * bb, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
            cusolverDnZgeqrf(sol, (int)rows, (int)bb, (cuDoubleComplex*)A_, (int)rows, (cuDoubleComplex*)tau, work,
                             lwork, dinfo) != CUSOLVER_STATUS_SUCCESS ||
            cusolverDnZungqr(sol, (int)rows, (int)bb, (int)bb, (cuDoubleComplex*)A_, (int)rows,
                             (const cuDoubleComplex*)tau, work, lwork, dinfo) != CUSOLVER_STATUS_SUCCESS ||
            cudaMemcpyAsync(&hinfo, dinfo, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
          rc = fail(CMPS_ERR_SOLVER, "randomized SVD: Householder QR failed");
          return;
        }
        if (hinfo != 0)
          qr_unrecovered = true;
        else if (cudaMemsetAsync(chol_bad, 0, sizeof(int), st) != cudaSuccess)
          rc = fail(CMPS_ERR_CUDA, "randomized SVD: QR flag reset failed");
      };
      if (rc == CMPS_OK) cudaMemsetAsync(chol_bad, 0, sizeof(int), st);
      if (rc == CMPS_OK) k_fill_random<<<grid_of(ll * bb), 256, 0, st>>>(Z, ll * bb, 0x5eed5eedull + (uint64_t)m);
      zg(opM, CUBLAS_OP_N, pp, bb, ll, &one, dA, nr, Z, ll, &zero, Y, pp);  // Y = M Omega
      qr(Y, pp);
      for (int it = 0; it < kRandIters; ++it) {
        zg(opMH, CUBLAS_OP_N, ll, bb, pp, &one, dA, nr, Y, pp, &zero, Z, ll);  // Z = M^H Q
        qr(Z, ll);
        zg(opM, CUBLAS_OP_N, pp, bb, ll, &one, dA, nr, Z, ll, &zero, Y, pp);   // Y = M Z
        qr(Y, pp);
      }
      // every QR of the range finder resets the flag: an unrepaired breakdown sets it again
      if (rc == CMPS_OK && qr_unrecovered && cudaMemsetAsync(chol_bad, 0x01, sizeof(int), st) != cudaSuccess)
        rc = fail(CMPS_ERR_CUDA, "randomized SVD: QR flag failed");
      zg(opMH, CUBLAS_OP_N, ll, bb, pp, &one, dA, nr, Y, pp, &zero, Z, ll);    // Z = M^H Q = B^H
      if (rc == CMPS_OK && cudaMemcpyAsync(Z2, Z, sizeof(double2) * ll * bb, cudaMemcpyDeviceToDevice, st) !=
                               cudaSuccess)
        rc = fail(CMPS_ERR_CUDA, "randomized SVD copy failed");
      int info = 0;
      if (!b.red_exact) {
        // The reduced problem by the Hermitian eigensolver: B B^H = U_r S^2 U_r^H,
        // B = U_r S (B^H U_r S^-1)^H.  Small values carry the Gram error
        // eps s_0^2 / s_j, which check (4) of the selection bounds; a sector
        // that fails it is redone with the reduced SVD below.
        zg(CUBLAS_OP_C, CUBLAS_OP_N, bb, bb, ll, &one, Z, ll, Z, ll, &zero, Gb, bb);
        if (rc == CMPS_OK && cusolverDnZheevd(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, (int)bb,
                                              (cuDoubleComplex*)Gb, (int)bb, W, work, lwork, dinfo) !=
                                 CUSOLVER_STATUS_SUCCESS)
          rc = fail(CMPS_ERR_SOLVER, "randomized SVD: reduced eigensolver failed");
        std::vector<double> w(bb);
        if (rc == CMPS_OK) {
          cudaMemcpyAsync(w.data(), W, sizeof(double) * bb, cudaMemcpyDeviceToHost, st);
          cudaMemcpyAsync(&info, dinfo, sizeof(int), cudaMemcpyDeviceToHost, st);
          if (cudaStreamSynchronize(st) != cudaSuccess || info != 0)
            rc = fail(CMPS_ERR_SOLVER, "randomized SVD: reduced eigensolver did not converge");
        }
        if (rc == CMPS_OK) {
          b.s.assign(bb, 0.0);
          for (int64_t j = 0; j < bb; ++j) b.s[j] = std::sqrt(std::max(0.0, w[bb - 1 - j]));
          rc = copy_wait(dS, b.s.data(), sizeof(double) * bb, cudaMemcpyHostToDevice, st);
        }
        if (rc == CMPS_OK) {
          k_reverse_cols<<<grid_of(bb * bb), 256, 0, st>>>(Gb, bb, R);  // U_r, descending
          double2* F = left ? b.dU : b.dV;   // short-side vectors (ld pp)
          double2* O = left ? b.dV : b.dU;   // long-side vectors (ld ll)
          zg(CUBLAS_OP_N, CUBLAS_OP_N, pp, bb, bb, &one, Y, pp, R, bb, &zero, F, pp);   // F = Q U_r
          zg(CUBLAS_OP_N, CUBLAS_OP_N, ll, bb, bb, &one, Z, ll, R, bb, &zero, O, ll);   // O = B^H U_r
          if (rc == CMPS_OK) k_scale_cols_inv<<<grid_of(ll * bb), 256, 0, st>>>(O, ll, bb, dS);  // ... S^-1
        }
      }
      // B^H = Q_B R (Householder), R^H = U_r S V_r^H, so B = U_r S (Q_B V_r)^H
      if (b.red_exact && rc == CMPS_OK &&
          cusolverDnZgeqrf(sol, (int)ll, (int)bb, (cuDoubleComplex*)Z, (int)ll, (cuDoubleComplex*)tau,
                                            work, lwork, dinfo) != CUSOLVER_STATUS_SUCCESS)
        rc = fail(CMPS_ERR_SOLVER, "randomized SVD QR failed");
      if (b.red_exact && rc == CMPS_OK) k_upper_adjoint<<<grid_of(bb * bb), 256, 0, st>>>(Z, ll, bb, Gb);
      if (b.red_exact && rc == CMPS_OK && cusolverDnZungqr(sol, (int)ll, (int)bb, (int)bb, (cuDoubleComplex*)Z, (int)ll,
                                            (const cuDoubleComplex*)tau, work, lwork, dinfo) != CUSOLVER_STATUS_SUCCESS)
        rc = fail(CMPS_ERR_SOLVER, "randomized SVD QR basis failed");
      if (b.red_exact && rc == CMPS_OK && cusolverDnZgesvdj(sol, CUSOLVER_EIG_MODE_VECTOR, 1, (int)bb, (int)bb, (cuDoubleComplex*)Gb,
                                             (int)bb, dS, (cuDoubleComplex*)R, (int)bb, (cuDoubleComplex*)Vb, (int)bb,
                                             work, lwork, dinfo, fw.params) != CUSOLVER_STATUS_SUCCESS)
        rc = fail(CMPS_ERR_SOLVER, "randomized SVD of the reduced matrix failed");
      if (b.red_exact && rc == CMPS_OK) {
        b.s.assign(bb, 0.0);
        cudaMemcpyAsync(b.s.data(), dS, sizeof(double) * bb, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(&info, dinfo, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess || info < 0)
          rc = fail(CMPS_ERR_SOLVER, "randomized SVD: reduced SVD failed");
      }
      if (rc == CMPS_OK) {
        double2* F = left ? b.dU : b.dV;   // short-side vectors (ld pp)
        double2* O = left ? b.dV : b.dU;   // long-side vectors (ld ll)
        if (b.red_exact) {
          zg(CUBLAS_OP_N, CUBLAS_OP_N, pp, bb, bb, &one, Y, pp, R, bb, &zero, F, pp);   // F = Q U_r
          zg(CUBLAS_OP_N, CUBLAS_OP_N, ll, bb, bb, &one, Z, ll, Vb, bb, &zero, O, ll);  // O = Q_B V_r
        }
        zg(opM, CUBLAS_OP_N, pp, bb, ll, &one, dA, nr, O, ll, &zero, R, pp);     // M O
        if (rc == CMPS_OK) k_col_resid<<<(unsigned)bb, 256, 0, st>>>(R, F, dS, pp, rs);
        // A <- A - Q Q^H A (left) or A - A Q Q^H (tall): the part outside the range
        if (left)
          zg(CUBLAS_OP_N, CUBLAS_OP_C, nr, nc, bb, &mone, Y, nr, Z2, nc, &one, dA, nr);
        else
          zg(CUBLAS_OP_N, CUBLAS_OP_C, nr, nc, bb, &mone, Z2, nr, Y, nc, &one, dA, nr);
        if (rc == CMPS_OK) {
          k_sumsq_partial<<<kSumBlocks, 256, 0, st>>>(dA, nr * nc, part);
          k_sum_final<<<1, 32, 0, st>>>(part, kSumBlocks, tailp);
          std::vector<double> r2(bb);
          double tail = 0.0;
          int bad = 0;
          cudaMemcpyAsync(r2.data(), rs, sizeof(double) * bb, cudaMemcpyDeviceToHost, st);
          cudaMemcpyAsync(&tail, tailp, sizeof(double), cudaMemcpyDeviceToHost, st);
          cudaMemcpyAsync(&bad, chol_bad, sizeof(int), cudaMemcpyDeviceToHost, st);
          if (cudaStreamSynchronize(st) != cudaSuccess) rc = fail(CMPS_ERR_CUDA, "randomized SVD failed");
          b.resid.assign(bb, 0.0);
          for (int64_t j = 0; j < bb; ++j) b.resid[j] = std::sqrt(std::max(0.0, r2[j]));
          // a broken-down factorisation leaves no usable basis: an infinite
          // tail fails the selection's check and sends the sector to the Gram route
          b.tail = bad ? HUGE_VAL : tail;
        }
      }
      if (ownW) dfree(work);
      if (ownX) dfree(X);
      if (rc == CMPS_OK) {
        b.eig = true;
        b.rnd = true;
      }
      return rc;
    };
    // mode 0: randomized route where eligible, else by size; 1: Gram route
    // for sectors of at least kEigMin, else exact; 2: exact; 3: randomized
    // route with blk[m].bb triplets (a wider range than mode 0's)
    auto factor = [&](int m, int mode, FW& fw) -> int {
      const cudaStream_t st = fw.st;
      const cusolverDnHandle_t sol = fw.sol;
      const cublasHandle_t blas = fw.blas;
      const gesvdjInfo_t params = fw.params;
      double2* const dA = fw.dA;
      double* const dS = fw.dS;
      int* const dinfo = fw.dinfo;
      Blk& b = blk[m];
      const int64_t C = th.ncols[m];
      const double* bre = H.theta.re() + th.base[m];
      const double* bim = H.theta.im() + th.base[m];
      const int64_t nr = (int64_t)b.rows.size(), nc = (int64_t)b.cols.size();
      const int64_t mn = std::min(nr, nc);
      k_gather_cm<<<grid_of(nr * nc), 256, 0, st>>>(bre, bim, C, b.drows, nr, b.dcols, nc, dA);
      b.rnd = false;
      b.tail = 0.0;
      b.resid.clear();
      if (mode == 0 && rand_b(m, mn) > 0) {
        b.bb = rand_b(m, mn);
        return factor_rand(m, b.bb, fw);
      }
      if (mode == 3) return factor_rand(m, b.bb, fw);
      b.s.resize(mn);
      if (mode == 2 || mn < kEigMin) {
        b.eig = false;
        int lwork = 0;
        if (cusolverDnZgesvdj_bufferSize(sol, CUSOLVER_EIG_MODE_VECTOR, 1, (int)nr, (int)nc, (cuDoubleComplex*)dA,
                                         (int)nr, dS, (cuDoubleComplex*)b.dU, (int)nr, (cuDoubleComplex*)b.dV,
                                         (int)nc, &lwork, params) != CUSOLVER_STATUS_SUCCESS)
          return fail(CMPS_ERR_SOLVER, "gesvdj buffer query failed");
        cuDoubleComplex* work = fw.work;
        const bool own = (size_t)lwork > fw.workcap;
        if (own && dmalloc(&work, sizeof(cuDoubleComplex) * std::max(1, lwork)) != cudaSuccess)
          return fail(CMPS_ERR_NOMEM, "SVD work allocation failed");
        cusolverStatus_t cs = cusolverDnZgesvdj(sol, CUSOLVER_EIG_MODE_VECTOR, 1, (int)nr, (int)nc,
                                                (cuDoubleComplex*)dA, (int)nr, dS, (cuDoubleComplex*)b.dU, (int)nr,
                                                (cuDoubleComplex*)b.dV, (int)nc, work, lwork, dinfo, params);
        int info = 0;
        cudaMemcpyAsync(b.s.data(), dS, sizeof(double) * mn, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(&info, dinfo, sizeof(int), cudaMemcpyDeviceToHost, st);
        cudaError_t ce = cudaStreamSynchronize(st);
        if (own) dfree(work);
        if (cs != CUSOLVER_STATUS_SUCCESS || ce != cudaSuccess) return fail(CMPS_ERR_SOLVER, "gesvdj failed");
        if (info < 0) return fail(CMPS_ERR_SOLVER, "gesvdj: invalid argument");
        return CMPS_OK;  // info > 0: not converged to tolerance within max sweeps; values still usable
      }
      b.eig = true;
      const bool left = nr <= nc;  // eigenvectors of A A^H give U; of A^H A give V
      const int p = (int)(left ? nr : nc);
      const bool ownG = (size_t)p * p > fw.Gcap || (size_t)p > fw.Wcap;
      double2* G = ownG ? nullptr : fw.G;   // Gram matrix, then its eigenvectors
      double* W = ownG ? nullptr : fw.W;
      int lwork = 0;
      if (ownG && (dmalloc(&G, sizeof(double2) * (size_t)p * p) != cudaSuccess ||
                   dmalloc(&W, sizeof(double) * p) != cudaSuccess)) {
        if (G) dfree(G);
        return fail(CMPS_ERR_NOMEM, "Gram matrix allocation failed");
      }
      const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
      cublasStatus_t bs;
      if (left)
        bs = cublasZgemm(blas, CUBLAS_OP_N, CUBLAS_OP_C, p, p, (int)nc, &one, (cuDoubleComplex*)dA, (int)nr,
                         (cuDoubleComplex*)dA, (int)nr, &zero, (cuDoubleComplex*)G, p);
      else
        bs = cublasZgemm(blas, CUBLAS_OP_C, CUBLAS_OP_N, p, p, (int)nr, &one, (cuDoubleComplex*)dA, (int)nr,
                         (cuDoubleComplex*)dA, (int)nr, &zero, (cuDoubleComplex*)G, p);
      int rc = CMPS_OK;
      cuDoubleComplex* work = nullptr;
      if (bs != CUBLAS_STATUS_SUCCESS) rc = fail(CMPS_ERR_CUDA, "Gram matrix GEMM failed");
      if (rc == CMPS_OK && cusolverDnZheevd_bufferSize(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, p,
                                                       (cuDoubleComplex*)G, p, W, &lwork) != CUSOLVER_STATUS_SUCCESS)
        rc = fail(CMPS_ERR_SOLVER, "zheevd buffer query failed");
      const bool ownW = (size_t)lwork > fw.workcap;
      if (!ownW) work = fw.work;
      if (rc == CMPS_OK && ownW && dmalloc(&work, sizeof(cuDoubleComplex) * std::max(1, lwork)) != cudaSuccess)
        rc = fail(CMPS_ERR_NOMEM, "zheevd work allocation failed");
      if (rc == CMPS_OK && cusolverDnZheevd(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, p,
                                            (cuDoubleComplex*)G, p, W, work, lwork, dinfo) != CUSOLVER_STATUS_SUCCESS)
        rc = fail(CMPS_ERR_SOLVER, "zheevd failed");
      std::vector<double> w(p);
      int info = 0;
      if (rc == CMPS_OK) {
        cudaMemcpyAsync(w.data(), W, sizeof(double) * p, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(&info, dinfo, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess || info != 0) rc = fail(CMPS_ERR_SOLVER, "zheevd did not converge");
      }
      if (rc == CMPS_OK) {
        for (int j = 0; j < p; ++j) b.s[j] = std::sqrt(std::max(0.0, w[p - 1 - j]));
        cudaMemcpyAsync(dS, b.s.data(), sizeof(double) * p, cudaMemcpyHostToDevice, st);
        double2* F = left ? b.dU : b.dV;   // the factor from the eigenvectors, descending order
        double2* O = left ? b.dV : b.dU;   // the other factor
        k_reverse_cols<<<grid_of((int64_t)p * p), 256, 0, st>>>(G, p, F);
        if (left)  // V = A^H U S^-1
          bs = cublasZgemm(blas, CUBLAS_OP_C, CUBLAS_OP_N, (int)nc, p, (int)nr, &one, (cuDoubleComplex*)dA, (int)nr,
                           (cuDoubleComplex*)F, (int)nr, &zero, (cuDoubleComplex*)O, (int)nc);
        else       // U = A V S^-1
          bs = cublasZgemm(blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)nr, p, (int)nc, &one, (cuDoubleComplex*)dA, (int)nr,
                           (cuDoubleComplex*)F, (int)nc, &zero, (cuDoubleComplex*)O, (int)nr);
        if (bs != CUBLAS_STATUS_SUCCESS) rc = fail(CMPS_ERR_CUDA, "second factor GEMM failed");
        k_scale_cols_inv<<<grid_of((left ? nc : nr) * (int64_t)p), 256, 0, st>>>(O, left ? nc : nr, p, dS);
        if (cudaStreamSynchronize(st) != cudaSuccess) rc = fail(CMPS_ERR_CUDA, "eigen-route SVD failed");
      }
      if (work && ownW) dfree(work);
      if (ownG) {
        dfree(G);
        dfree(W);
      }
      return rc;
    };
    FW main_fw{st, sol, blas, params, dA, dS, dinfo};
    std::vector<int> todo;
    int n_eig = 0;
    for (int m = 0; m < nm; ++m) {
      if (blk[m].rows.empty()) continue;
      todo.push_back(m);
      if (std::min(blk[m].rows.size(), blk[m].cols.size()) >= (size_t)kEigMin) ++n_eig;
    }
    // Concurrent factoring when at least two sectors take the Gram route:
    // sectors dealt largest first to the least-loaded worker, one host thread
    // per worker, workspaces sized for the worker's largest sector and
    // bounded in total; otherwise the sectors run one by one.
    bool done = false;
    SvdPool* pool = nullptr;
    const bool have_pool = get_pool(H.ctx, &pool) == CMPS_OK;  // set up on the first SVD, whatever its size
    if (n_eig >= 2 && have_pool) {
      int K = std::min<int>((int)pool->w.size(), (int)todo.size());
      // One queue, longest sectors first; each worker takes the next sector
      // when it is free.  Estimated milliseconds per route (measured on
      // B200): the randomized route is bound by its FP64 GEMMs, the Gram
      // route and the one-sided Jacobi SVD by their sequential sweeps.
      std::vector<int> order = todo;
      auto cost = [&](int m) {
        const double nr = (double)blk[m].rows.size(), nc = (double)blk[m].cols.size();
        const int64_t mn = (int64_t)std::min(nr, nc);
        if (rand_b(m, mn) > 0) return 10.0 + 2e-8 * nr * nc * (double)rand_b(m, mn);
        if (mn >= kEigMin) return 0.013 * (double)mn + 2.5e-9 * (double)mn * (double)mn * (double)mn;
        return 0.1 + 0.09 * (double)mn;
      };
      std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost(x) > cost(y); });
      std::vector<FW> fws(K);
      std::vector<size_t> nA(K, 1), nS(K, 1), nG(K, 0), nW(K, 0), nX(K, 0), nwork(K, 1);
      bool ok = true;
      for (int k = 0; k < K && ok; ++k) {
        SvdWorker& w = pool->w[k];
        fws[k] = FW{w.st, w.sol, w.blas, nullptr, nullptr, nullptr, nullptr};
        if (cusolverDnCreateGesvdjInfo(&fws[k].params) != CUSOLVER_STATUS_SUCCESS) {
          fws[k].params = nullptr;
          ok = false;
          break;
        }
        cusolverDnXgesvdjSetTolerance(fws[k].params, 0.0);
        cusolverDnXgesvdjSetMaxSweeps(fws[k].params, 100);
        cusolverDnXgesvdjSetSortEig(fws[k].params, 1);
        for (int m : order) {  // any worker may take any sector
          const int64_t nr = (int64_t)blk[m].rows.size(), nc = (int64_t)blk[m].cols.size();
          const int64_t mn = std::min(nr, nc);
          nA[k] = std::max(nA[k], (size_t)(nr * nc));
          nS[k] = std::max(nS[k], (size_t)mn);
          int lwork = 0;
          if (rand_b(m, mn) > 0) {
            nX[k] = std::max(nX[k], rand_scratch(nr, nc, rand_b(m, mn)));
            if (rand_lwork(w.sol, fws[k].params, std::max(nr, nc), rand_b(m, mn), &lwork) != CMPS_OK) ok = false;
          } else if (mn < kEigMin) {
            if (cusolverDnZgesvdj_bufferSize(w.sol, CUSOLVER_EIG_MODE_VECTOR, 1, (int)nr, (int)nc,
                                             (cuDoubleComplex*)dA, (int)nr, dS, (cuDoubleComplex*)blk[m].dU, (int)nr,
                                             (cuDoubleComplex*)blk[m].dV, (int)nc, &lwork,
                                             fws[k].params) != CUSOLVER_STATUS_SUCCESS)
              ok = false;
          } else {
            const int pp = (int)mn;
            nG[k] = std::max(nG[k], (size_t)pp * pp);
            nW[k] = std::max(nW[k], (size_t)pp);
            if (cusolverDnZheevd_bufferSize(w.sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, pp,
                                            (cuDoubleComplex*)dA, pp, dS, &lwork) != CUSOLVER_STATUS_SUCCESS)
              ok = false;
          }
          nwork[k] = std::max(nwork[k], (size_t)std::max(1, lwork));
        }
      }
      // every worker is sized for any sector: as many workers as 8 GB of
      // workspace allows (fewer than two: the sequential path)
      double bytes = 0.0;
      for (int k = 0; k < K; ++k)
        bytes += 16.0 * (nA[k] + nG[k] + nX[k] + nwork[k]) + 8.0 * (nS[k] + nW[k]) + 4.0;
      if (bytes > 8e9) {
        const double per = bytes / K;
        K = std::min<int>(K, (int)(8e9 / per));
        bytes = per * K;
      }
      if (ok && K >= 2 && bytes <= 8e9) {
        for (int k = 0; k < K && ok; ++k) {
          FW& fw = fws[k];
          if (dmalloc(&fw.dA, sizeof(double2) * nA[k]) != cudaSuccess ||
              dmalloc(&fw.dS, sizeof(double) * nS[k]) != cudaSuccess ||
              dmalloc(&fw.dinfo, sizeof(int)) != cudaSuccess ||
              dmalloc(&fw.work, sizeof(cuDoubleComplex) * nwork[k]) != cudaSuccess ||
              (nG[k] && dmalloc(&fw.G, sizeof(double2) * nG[k]) != cudaSuccess) ||
              (nW[k] && dmalloc(&fw.W, sizeof(double) * nW[k]) != cudaSuccess) ||
              (nX[k] && dmalloc(&fw.X, sizeof(double2) * nX[k]) != cudaSuccess)) {
            ok = false;
            break;
          }
          fw.workcap = nwork[k];
          fw.Gcap = nG[k];
          fw.Wcap = nW[k];
          fw.Xcap = nX[k];
        }
        if (ok) {
          // theta and the block descriptors were written on the handle's stream
          cudaStreamSynchronize(st);
          std::vector<int> code(K, CMPS_OK);
          std::vector<std::string> msg(K);
          std::vector<std::thread> th_w;
          std::atomic<size_t> next{0};
          const int dev = H.ctx->device;
          for (int k = 0; k < K; ++k)
            th_w.emplace_back([&, k]() {
              cudaSetDevice(dev);
              for (;;) {
                const size_t i = next.fetch_add(1);
                if (i >= order.size() || code[k] != CMPS_OK) break;
                const auto t0 = std::chrono::steady_clock::now();
                const int rc = factor(order[i], 0, fws[k]);
                if (std::getenv("CMPS_SVD_TRACE")) {
                  cudaStreamSynchronize(fws[k].st);
                  const Blk& bk = blk[order[i]];
                  std::fprintf(stderr, "svd sector %d (%zu x %zu) route %s b=%lld: %.2f ms (worker %d)\n", order[i],
                               bk.rows.size(), bk.cols.size(), bk.rnd ? "rnd" : bk.eig ? "gram" : "exact",
                               (long long)bk.bb,
                               std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count(),
                               k);
                }
                if (rc != CMPS_OK) {
                  code[k] = rc;
                  msg[k] = cmps_last_error();
                  next.store(order.size());  // the others stop after their current sector
                }
              }
              cudaStreamSynchronize(fws[k].st);
            });
          for (auto& t : th_w) t.join();
          for (int k = 0; k < K; ++k)
            if (code[k] != CMPS_OK && status == CMPS_OK) status = fail(code[k], msg[k]);
          done = true;
        }
      }
      for (FW& fw : fws) {
        if (fw.dA) dfree(fw.dA);
        if (fw.dS) dfree(fw.dS);
        if (fw.dinfo) dfree(fw.dinfo);
        if (fw.work) dfree(fw.work);
        if (fw.G) dfree(fw.G);
        if (fw.W) dfree(fw.W);
        if (fw.X) dfree(fw.X);
        if (fw.params) cusolverDnDestroyGesvdjInfo(fw.params);
      }
    }
    if (!done)
      for (int m : todo) {
        if (status != CMPS_OK) break;
        status = factor(m, 0, main_fw);
      }
    // ---- global selection ----
    // Sectors of the randomized route contribute only their leading values.
    // Their result stands when it settles the truncation of the whole
    // spectrum: (1) the kept count is decided inside the computed values,
    // with a margin of 1 % on the trailing weight (computed values plus the
    // sectors' tails): by the bond-dimension cap (the weight from index
    // cap - 1 on is at least 1.01 max_trunc), or else by the weight cut (the
    // rule's loop from the end, run over the computed values with the tails
    // as the last weight, stops inside them, on a weight at least 1.01
    // max_trunc whose predecessor is at most 0.99 max_trunc; a cut that close
    // to the threshold goes to the Gram route at once); (2) the degeneracy
    // extension ends inside the computed values; (3) no value left out can rank above
    // the first discarded one (each sector's tail, which bounds its largest
    // value left out, is below half of it); (4) every kept triplet has
    // converged: residual <= 1e-12 s_0 + 500 eps s_0^2 / s_j, the second term
    // being the error the Gram matrix itself leaves in a vector of value s_j.
    // Otherwise those sectors are redone
    // by the Gram route.  Gram-route sectors are redone exactly where that
    // route is not accurate enough (weight-decided count, or a kept value
    // below 1e-5 s_0).
    struct SV { double v; int m; int64_t j; };
    std::vector<SV> all;
    std::vector<double> sv;
    int64_t length = 0;
    double tail_total = 0.0;
    bool settled = false;
    // Passes: at most one to make the values exact for a weight cut, one per
    // doubling of a randomized range (six from 64 triplets in an 8192-wide
    // sector), one to the Gram route, one to redo it exactly, one to settle.
    for (int pass = 0; pass < 12 && status == CMPS_OK && !settled; ++pass) {
      all.clear();
      int64_t n_true = 0;
      bool any_rnd = false;
      tail_total = 0.0;
      for (int m = 0; m < nm; ++m) {
        for (int64_t j = 0; j < (int64_t)blk[m].s.size(); ++j) all.push_back(SV{blk[m].s[j], m, j});
        if (!blk[m].rows.empty()) n_true += (int64_t)std::min(blk[m].rows.size(), blk[m].cols.size());
        if (blk[m].rnd) {
          any_rnd = true;
          tail_total += blk[m].tail;
        }
      }
      if (all.empty()) { status = fail(CMPS_ERR_SOLVER, "no singular values (empty wavefunction)"); break; }
      std::stable_sort(all.begin(), all.end(), [](const SV& a, const SV& b) { return a.v > b.v; });
      sv.assign(all.size(), 0.0);
      for (size_t i = 0; i < all.size(); ++i) sv[i] = all[i].v;
      bool weight_decided = false;
      if (any_rnd) {
        const int64_t np = (int64_t)sv.size();
        const int64_t cap = (chi > 0 && chi < n_true) ? chi : n_true;
        bool valid = sv[0] > 0.0;
        // which check failed (CMPS_SVD_TRACE); 5: a weight cut within the margin, 6: a
        // weight cut read from eigensolver values
        int failed = valid ? 0 : 0x10;
        int64_t len = cap;
        if (valid) {
          double beyond = tail_total;
          const bool cap_inside = cap < n_true && cap + 1 < np;
          if (cap_inside)
            for (int64_t i = cap - 1; i < np; ++i) beyond += sv[i] * sv[i];
          bool exact_values = true;  // every value of the sectors involved has an absolute error ~eps s_0
          for (int m = 0; m < nm; ++m)
            if (!blk[m].rows.empty() && blk[m].eig && (blk[m].rnd ? !blk[m].red_exact : true)) exact_values = false;
          if (!(cap_inside && beyond >= 1.01 * max_trunc)) {                   // (1), weight cut
            if (!(tail_total < max_trunc)) {
              // the weight left out reaches the threshold by itself: the cut
              // lies beyond the computed values, and only a wider range can
              // settle it
              valid = false;
              failed = 1;
            } else if (!exact_values) {
              // values of an eigensolver (the reduced one, or the Gram
              // route's) carry ~eps s_0^2 on every s_j^2, which can exceed a
              // small threshold by itself: first the same sectors exactly
              valid = false;
              failed = 6;
            } else {
              // truncation_length's loop, the tails standing for the values
              // left out (all of them rank below the cut: check (3)).  The
              // margin covers the error of the partial weights: ~2 eps s_0 s_j
              // on each s_j^2, and the rounding of the tails.
              double err = tail_total, before = tail_total, ssum = 0.0, entries = 0.0;
              int64_t tl = np;
              while (err < max_trunc && tl > 0) {
                before = err;
                err += sv[tl - 1] * sv[tl - 1];
                ssum += sv[tl - 1];
                --tl;
              }
              for (int m = 0; m < nm; ++m)
                if (blk[m].rnd) entries += (double)blk[m].rows.size() * (double)blk[m].cols.size();
              const double slack = std::max(0.01 * max_trunc, 64.0 * kEps * sv[0] * ssum +
                                                                  64.0 * kEps * kEps * sv[0] * sv[0] * entries);
              const bool clear = err < max_trunc ? err <= max_trunc - slack
                                                 : err >= max_trunc + slack && before <= max_trunc - slack;
              len = tl + 1;
              if (len >= cap || len >= np) {
                valid = false;
                failed = 1;
              } else if (!clear) {
                valid = false;
                failed = 5;
              } else {
                weight_decided = true;
              }
            }
          }
        }
        if (valid) {
          while (len < n_true && len < np && (sv[len - 1] - sv[len]) / sv[len - 1] < 1.0e-3) ++len;
          valid = len < np;                                                     // (2)
          if (!valid) failed = 2;
        }
        std::vector<char> bad4(nm, 0);  // sectors whose kept triplets miss check (4)
        if (valid) {
          const double next = sv[len];
          std::vector<int64_t> kept(nm, 0);
          for (int64_t g = 0; g < len; ++g) kept[all[g].m] = std::max(kept[all[g].m], all[g].j + 1);
          for (int m = 0; m < nm && valid; ++m) {
            if (!blk[m].rnd) continue;
            if (!(4.0 * blk[m].tail < next * next)) valid = false, failed = 3;  // (3)
          }
          for (int m = 0; m < nm && valid; ++m) {
            if (!blk[m].rnd) continue;
            for (int64_t j = 0; j < kept[m] && !bad4[m]; ++j)
              if (!(blk[m].resid[j] <= 1e-12 * sv[0] + 500.0 * kEps * sv[0] * sv[0] / blk[m].s[j]))
                bad4[m] = 1;                                                    // (4)
          }
          for (int m = 0; m < nm && valid; ++m)
            if (bad4[m]) valid = false, failed = 4;
        }
        if (std::getenv("CMPS_SVD_TRACE")) {
          std::fprintf(stderr, "svd pass %d: randomized %s (check %d)", pass, valid ? "accepted" : "rejected", failed);
          for (int m = 0; m < nm; ++m)
            if (blk[m].rnd)
              std::fprintf(stderr, "  [m%d b=%lld tail=%.3g]", m, (long long)blk[m].bb, blk[m].tail);
          std::fprintf(stderr, "\n");
        }
        if (!valid && failed == 6) {
          // a weight cut read from eigensolver values: the randomized
          // sectors again with the reduced SVD (same range), the Gram-route
          // ones with the one-sided Jacobi SVD
          for (int m = 0; m < nm && status == CMPS_OK; ++m) {
            if (blk[m].rows.empty() || !blk[m].eig) continue;
            if (blk[m].rnd) {
              if (blk[m].red_exact) continue;
              blk[m].red_exact = true;
              status = factor(m, 3, main_fw);
            } else {
              status = factor(m, 2, main_fw);
            }
          }
          continue;
        }
        if (!valid && failed == 4) {
          // kept triplets of the reduced eigensolver not accurate enough:
          // those sectors again with the reduced SVD (QR + one-sided Jacobi),
          // same range
          bool retried = false;
          for (int m = 0; m < nm && status == CMPS_OK; ++m) {
            if (!bad4[m] || blk[m].red_exact) continue;
            blk[m].red_exact = true;
            status = factor(m, 3, main_fw);
            retried = true;
          }
          if (retried) continue;
        }
        if (!valid) {
          // A spectrum that decays slowly past the range leaves too much
          // tail (check 3): widen the range (twice the triplets) while it
          // stays well under the sector's short side, else take the Gram
          // route.  Both cost far less than the one-sided Jacobi SVD that
          // the Gram route falls back to for kept values below 1e-5 s_0.
          // A cut within 1 % of the threshold (check 5) depends on rounding
          // the range cannot remove: the Gram route at once.
          for (int m = 0; m < nm && status == CMPS_OK; ++m) {
            if (!blk[m].rnd) continue;
            const int64_t mn = std::min(blk[m].rows.size(), blk[m].cols.size());
            if (failed != 5 && 4 * (2 * blk[m].bb) <= 3 * mn) {
              blk[m].bb *= 2;
              status = factor(m, 3, main_fw);
            } else {
              status = factor(m, 1, main_fw);
            }
          }
          continue;
        }
        length = len;
      } else {
        length = truncation_length(sv, chi, max_trunc, &weight_decided);
      }
      const double floor2 = 1e-10 * sv[0] * sv[0];
      bool redo = false;
      for (int m = 0; m < nm; ++m) {
        if (!blk[m].eig || blk[m].rnd) continue;  // the randomized route resolves small values directly
        bool low = false;
        for (int64_t g = 0; g < length; ++g)
          if (all[g].m == m && all[g].v * all[g].v < floor2) low = true;
        if (weight_decided || low) {
          redo = true;
          if ((status = factor(m, 2, main_fw)) != CMPS_OK) break;
        }
      }
      settled = !redo;
    }
    if (status == CMPS_OK && !settled) status = fail(CMPS_ERR_STATE, "SVD: truncation not settled");
    cusolverDnDestroyGesvdjInfo(params);
    if (status != CMPS_OK) break;
    out.values.assign(sv.begin(), sv.begin() + length);
    for (int m = 0; m < nm; ++m)
      if (!blk[m].rows.empty()) ++out.routes[blk[m].rnd ? 2 : blk[m].eig ? 1 : 0];
    out.discarded = tail_total;  // the weight the randomized sectors left out
    for (size_t i = length; i < sv.size(); ++i) out.discarded += sv[i] * sv[i];
    out.kept.assign(nm, 0);
    out.order.clear();
    for (int64_t g = 0; g < length; ++g) {
      out.order.push_back({all[g].m, all[g].j});
      out.kept[all[g].m] = std::max(out.kept[all[g].m], all[g].j + 1);
    }
    out.gidx.assign(nm, {});
    for (int m = 0; m < nm; ++m) out.gidx[m].assign(out.kept[m], -1);
    for (int64_t g = 0; g < length; ++g) out.gidx[all[g].m][all[g].j] = g;
    // ---- factors ----
    out.uoff.assign(nm, 0);
    out.voff.assign(nm, 0);
    int64_t ut = 0, vt = 0;
    for (int m = 0; m < nm; ++m) {
      out.uoff[m] = ut;
      out.voff[m] = vt;
      ut += th.nrows[m] * out.kept[m];
      vt += out.kept[m] * th.ncols[m];
    }
    if ((status = out.U.alloc(ut)) != CMPS_OK) break;
    if ((status = out.Vd.alloc(vt)) != CMPS_OK) break;
    if (ut) cudaMemsetAsync(out.U.d, 0, sizeof(double) * 2 * ut, st);
    if (vt) cudaMemsetAsync(out.Vd.d, 0, sizeof(double) * 2 * vt, st);
    for (int m = 0; m < nm; ++m) {
      const int64_t k = out.kept[m];
      if (k == 0) continue;
      Blk& b = blk[m];
      const int64_t nr = (int64_t)b.rows.size(), nc = (int64_t)b.cols.size();
      const int64_t mn = std::min(nr, nc);
      (void)mn;
      k_scatter_u<<<grid_of(nr * k), 256, 0, st>>>(b.dU, nr, k, b.drows, kEps / (double)nr, out.U.re() + out.uoff[m],
                                                   out.U.im() + out.uoff[m]);
      k_scatter_vd<<<grid_of(nc * k), 256, 0, st>>>(b.dV, nc, k, b.dcols, th.ncols[m], kEps / (double)nc,
                                                    out.Vd.re() + out.voff[m], out.Vd.im() + out.voff[m]);
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) { status = fail(CMPS_ERR_CUDA, "SVD scatter failed"); break; }
  } while (false);
  cleanup();
  return status;
}

// CheckConvergence (DMRG_routines.cpp:769-771) for a growth step:
// 1 - sum of the singular values of Aux diag(prev_lambda), where MakePrediction
// (:693-707) takes Aux = diag(s~) V~^dagger from the SVD of Lambda V^dagger
// reshaped to rows (sigma2, a1) and columns a2.  Aux^H Aux equals
// (Lambda V^dagger)^H (Lambda V^dagger), so the singular values of
// Aux diag(prev_lambda) are those of (Lambda V^dagger) diag(prev_lambda)
// itself; that matrix is block diagonal in the a2 charge, and each block's
// values come from a values-only one-sided Jacobi SVD (not the Gram matrix,
// whose small eigenvalues would carry an error ~ sqrt(eps) s_max).
int growth_fidelity(Heff& H, const SvdResult& s, const std::vector<double>& lam, const std::vector<double>& prev,
                    double* out) {
  const Rules& r = H.rules;
  const ThetaSpace& th = s.th;
  const Bond& A2 = s.a2;
  if ((int64_t)prev.size() != A2.size()) return fail(CMPS_ERR_STATE, "fidelity: previous values do not match the bond");
  cudaStream_t st = H.ctx->stream;
  cusolverDnHandle_t sol;
  CMPS_TRY(get_solver(H.ctx, &sol));
  gesvdjInfo_t params;
  if (cusolverDnCreateGesvdjInfo(&params) != CUSOLVER_STATUS_SUCCESS) return fail(CMPS_ERR_SOLVER, "gesvdj info");
  cusolverDnXgesvdjSetTolerance(params, 0.0);
  cusolverDnXgesvdjSetMaxSweeps(params, 100);
  double total = 0.0;
  int status = CMPS_OK;
  for (int t = 0; t < A2.nsec() && status == CMPS_OK; ++t) {
    const int64_t Cn = A2.sdim[t];
    std::vector<int64_t> src;
    std::vector<double> rs, cs(Cn);
    for (int64_t c = 0; c < Cn; ++c) cs[c] = prev[A2.selem[t][c]];
    for (int s2 = 0; s2 < H.d; ++s2) {
      const int m = th.find(r.sub(A2.sq[t], H.sigq[s2]));
      if (m < 0 || s.kept[m] == 0 || th.coloff[m][s2] < 0) continue;
      for (int64_t j = 0; j < s.kept[m]; ++j) {
        src.push_back(s.voff[m] + j * th.ncols[m] + th.coloff[m][s2]);
        rs.push_back(lam[s.gidx[m][j]]);
      }
    }
    const int64_t R = (int64_t)src.size();
    if (R == 0 || Cn == 0) continue;
    if (R > 0x7fffffff || Cn > 0x7fffffff) { status = fail(CMPS_ERR_ARG, "fidelity: block too large"); break; }
    int64_t* dsrc = nullptr;
    double *drs = nullptr, *dcs = nullptr, *dS = nullptr;
    double2 *dM = nullptr, *dU = nullptr, *dV = nullptr;
    cuDoubleComplex* work = nullptr;
    int* dinfo = nullptr;
    const int64_t mn = std::min(R, Cn);
    do {
      if (dmalloc(&dsrc, sizeof(int64_t) * R) != cudaSuccess || dmalloc(&drs, sizeof(double) * R) != cudaSuccess ||
          dmalloc(&dcs, sizeof(double) * Cn) != cudaSuccess || dmalloc(&dM, sizeof(double2) * R * Cn) != cudaSuccess ||
          dmalloc(&dS, sizeof(double) * mn) != cudaSuccess || dmalloc(&dU, sizeof(double2) * R * mn) != cudaSuccess ||
          dmalloc(&dV, sizeof(double2) * Cn * mn) != cudaSuccess || dmalloc(&dinfo, sizeof(int)) != cudaSuccess) {
        status = fail(CMPS_ERR_NOMEM, "fidelity: allocation failed");
        break;
      }
      if ((status = copy_wait(dsrc, src.data(), sizeof(int64_t) * R, cudaMemcpyHostToDevice, st)) != CMPS_OK) break;
      if ((status = copy_wait(drs, rs.data(), sizeof(double) * R, cudaMemcpyHostToDevice, st)) != CMPS_OK) break;
      if ((status = copy_wait(dcs, cs.data(), sizeof(double) * Cn, cudaMemcpyHostToDevice, st)) != CMPS_OK) break;
      k_gather_fid<<<grid_of(R * Cn), 256, 0, st>>>(s.Vd.re(), s.Vd.im(), dsrc, drs, dcs, R, Cn, dM);
      int lwork = 0;
      // the solver checks ldu >= rows and ldv >= columns even without vectors
      if (cusolverDnZgesvdj_bufferSize(sol, CUSOLVER_EIG_MODE_NOVECTOR, 1, (int)R, (int)Cn, (cuDoubleComplex*)dM,
                                       (int)R, dS, (cuDoubleComplex*)dU, (int)R, (cuDoubleComplex*)dV, (int)Cn,
                                       &lwork, params) != CUSOLVER_STATUS_SUCCESS) {
        status = fail(CMPS_ERR_SOLVER, "fidelity: gesvdj buffer query failed");
        break;
      }
      if (dmalloc(&work, sizeof(cuDoubleComplex) * std::max(1, lwork)) != cudaSuccess) {
        status = fail(CMPS_ERR_NOMEM, "fidelity: work allocation failed");
        break;
      }
      if (cusolverDnZgesvdj(sol, CUSOLVER_EIG_MODE_NOVECTOR, 1, (int)R, (int)Cn, (cuDoubleComplex*)dM, (int)R, dS,
                            (cuDoubleComplex*)dU, (int)R, (cuDoubleComplex*)dV, (int)Cn, work, lwork, dinfo,
                            params) != CUSOLVER_STATUS_SUCCESS) {
        status = fail(CMPS_ERR_SOLVER, "fidelity: gesvdj failed");
        break;
      }
      std::vector<double> sv(mn);
      if ((status = copy_wait(sv.data(), dS, sizeof(double) * mn, cudaMemcpyDeviceToHost, st)) != CMPS_OK) break;
      for (double v : sv) total += v;
    } while (false);
    dfree(dsrc);
    dfree(drs);
    dfree(dcs);
    dfree(dM);
    dfree(dS);
    dfree(dU);
    dfree(dV);
    dfree(work);
    dfree(dinfo);
  }
  cusolverDnDestroyGesvdjInfo(params);
  CMPS_TRY(status);
  *out = 1.0 - total;
  return CMPS_OK;
}

// CheckConvergence(Prediction, MPSDecomposition) (DMRG_routines.cpp:773-776),
// the fidelity of a finite sweep step: 1 - |<G, U diag(lam) V^dagger>|, G the
// predicted wavefunction the step's eigensolve started from (theta layout)
// and U diag(lam) V^dagger the new rescaled decomposition.  Per block m:
// P_m = U_m^H G_m (kept x ncols, one grouped GEMM), then the lam-weighted
// dot of P_m with V^dagger_m, summed on the host (both are chi x d chi).
int sweep_fidelity(Heff& H, const SvdResult& s, const std::vector<double>& lam, const Planar& guess, double* out) {
  const ThetaSpace& th = s.th;
  const int nm = (int)th.mq.size();
  if (guess.len != th.total) return fail(CMPS_ERR_STATE, "fidelity: guess is not in this theta layout");
  cudaStream_t st = H.ctx->stream;
  GemmPlan p;
  for (int m = 0; m < nm; ++m) {
    if (!s.kept[m]) continue;
    GemmTask t{};
    t.c_off = s.voff[m];  // P_m shares V^dagger_m's layout
    t.m = (int32_t)s.kept[m];
    t.n = (int32_t)th.ncols[m];
    t.ldc = (int32_t)th.ncols[m];
    t.t0 = (int32_t)p.terms.size();
    GemmTerm tm{};
    tm.a_off = s.uoff[m];  // U_m stored nrows x kept: op(A) = U_m^H
    tm.lda = (int32_t)s.kept[m];
    tm.k = (int32_t)th.nrows[m];
    tm.b_off = th.base[m];
    tm.ldb = (int32_t)th.ncols[m];
    p.terms.push_back(tm);
    t.t1 = (int32_t)p.terms.size();
    p.tasks.push_back(t);
  }
  double total_re = 0.0, total_im = 0.0;
  if (!p.tasks.empty()) {
    Planar P;
    CMPS_TRY(P.alloc(s.Vd.len));
    int rc = p.validate(true, false, s.U.len, guess.len, P.len, "fidelity");
    if (rc == CMPS_OK) rc = p.upload(st);
    if (rc == CMPS_OK) rc = launch_zgemm_fp64(p, true, false, s.U, guess, P, st);
    std::vector<double> hp(2 * (size_t)s.Vd.len), hv(2 * (size_t)s.Vd.len);
    if (rc == CMPS_OK) rc = copy_wait(hp.data(), P.d, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, st);
    if (rc == CMPS_OK) rc = copy_wait(hv.data(), s.Vd.d, sizeof(double) * hv.size(), cudaMemcpyDeviceToHost, st);
    p.release();
    P.release();
    CMPS_TRY(rc);
    const int64_t n = s.Vd.len;
    for (int m = 0; m < nm; ++m)
      for (int64_t j = 0; j < s.kept[m]; ++j) {
        const double w = lam[s.gidx[m][j]];
        for (int64_t k = 0; k < th.ncols[m]; ++k) {
          const int64_t o = s.voff[m] + j * th.ncols[m] + k;
          // conj(P) . Vd
          const double pr = hp[o], pi = hp[n + o], vr = hv[o], vi = hv[n + o];
          total_re += w * (pr * vr + pi * vi);
          total_im += w * (pr * vi - pi * vr);
        }
      }
  }
  *out = 1.0 - std::hypot(total_re, total_im);
  return CMPS_OK;
}

// New bond built from the kept singular vectors, in the reference's element
// order (descending singular value).
static void new_bond(const SvdResult& s, Bond& b, std::vector<int>& sec_of_m) {
  std::vector<QKey> q(s.order.size());
  for (size_t g = 0; g < s.order.size(); ++g) q[g] = s.th.mq[s.order[g].first];
  b.build(q);
  sec_of_m.assign(s.th.mq.size(), -1);
  for (size_t m = 0; m < s.th.mq.size(); ++m) sec_of_m[m] = s.kept[m] ? b.find(s.th.mq[m]) : -1;
}

static int alloc_env(const Rules& r, const Bond& a, int D, const std::vector<QKey>& bq, bool right, Env& env,
                     cudaStream_t st) {
  env.right = right;
  env.a = a;
  env.D = D;
  env.bq = bq;
  const int ns = a.nsec();
  env.off.assign((size_t)D * ns, -1);
  env.partner.assign((size_t)D * ns, -1);
  int64_t total = 0;
  for (int b = 0; b < D; ++b)
    for (int s = 0; s < ns; ++s) {
      int sp = a.find(r.add(a.sq[s], bq[b]));
      if (sp < 0) continue;
      env.partner[(size_t)b * ns + s] = sp;
      env.off[(size_t)b * ns + s] = total;
      total += a.sdim[s] * a.sdim[sp];
    }
  CMPS_TRY(env.data.alloc(total));
  return zero_wait(env.data.d, sizeof(double) * 2 * total, st);
}

int left_update(Heff& H, const SvdResult& s, Env& out) {
  const Rules& r = H.rules;
  const ThetaSpace& th = s.th;
  const int nm = (int)th.mq.size();
  const int d = H.d;
  const Bond& A0 = H.L.a;
  Bond nb;
  std::vector<int> sec;
  new_bond(s, nb, sec);
  CMPS_TRY(alloc_env(r, nb, H.D, H.bq, false, out, H.ctx->stream));
  // X^{b1}_m = LeftPart^{b1} U_m  (rows L(m'), cols kept[m])
  std::set<int> b1s;
  for (auto& kv : H.lp_off) b1s.insert(kv.first[0]);
  GemmPlan px, pl;
  std::vector<int64_t> xbase((size_t)H.D * nm, -1);
  int64_t xt = 0;
  for (int b1 : b1s)
    for (int m = 0; m < nm; ++m) {
      const int64_t k = s.kept[m];
      if (!k) continue;
      int mp = th.find(r.add(th.mq[m], H.bq[b1]));
      if (mp < 0 || !s.kept[mp]) continue;
      std::vector<GemmTask> tasks;
      std::vector<GemmTerm> terms;
      for (int s1p = 0; s1p < d; ++s1p) {
        if (th.rowoff[mp][s1p] < 0) continue;
        int sp = A0.find(r.sub(th.mq[mp], H.sigq[s1p]));
        GemmTask t{};
        t.c_off = th.rowoff[mp][s1p] * k;
        t.m = (int32_t)A0.sdim[sp];
        t.n = (int32_t)k;
        t.ldc = (int32_t)k;
        t.t0 = (int32_t)terms.size();
        for (int s1 = 0; s1 < d; ++s1) {
          if (th.rowoff[m][s1] < 0) continue;
          int sa = A0.find(r.sub(th.mq[m], H.sigq[s1]));
          auto it = H.lp_off.find({b1, s1p, s1, sa});
          if (it == H.lp_off.end()) continue;
          GemmTerm tm{};
          tm.a_off = it->second;
          tm.lda = (int32_t)A0.sdim[sa];
          tm.k = (int32_t)A0.sdim[sa];
          tm.b_off = s.uoff[m] + th.rowoff[m][s1] * k;
          tm.ldb = (int32_t)k;
          terms.push_back(tm);
        }
        t.t1 = (int32_t)terms.size();
        tasks.push_back(t);
      }
      if (terms.empty()) continue;
      int64_t xb = xt;
      xbase[(size_t)b1 * nm + m] = xb;
      xt += th.nrows[mp] * k;
      int32_t tb = (int32_t)px.terms.size();
      for (auto& tm : terms) px.terms.push_back(tm);
      for (auto& t : tasks) {
        t.c_off += xb;
        t.t0 += tb;
        t.t1 += tb;
        px.tasks.push_back(t);
      }
      // L'^{b1}: (kept[m'] x kept[m]) = U_{m'}^H X
      GemmTask lt{};
      const int ns = nb.nsec();
      lt.c_off = out.off[(size_t)b1 * ns + sec[m]];
      lt.m = (int32_t)s.kept[mp];
      lt.n = (int32_t)k;
      lt.ldc = (int32_t)k;
      lt.t0 = (int32_t)pl.terms.size();
      GemmTerm tm{};
      tm.a_off = s.uoff[mp];
      tm.lda = (int32_t)s.kept[mp];
      tm.k = (int32_t)th.nrows[mp];
      tm.b_off = xb;
      tm.ldb = (int32_t)k;
      pl.terms.push_back(tm);
      lt.t1 = (int32_t)pl.terms.size();
      pl.tasks.push_back(lt);
    }
  Planar X;
  CMPS_TRY(X.alloc(xt));
  int status = CMPS_OK;
  do {
    if ((status = px.validate(false, false, H.LP.len, s.U.len, xt, "left update X")) != CMPS_OK) break;
    if ((status = pl.validate(true, false, s.U.len, xt, out.data.len, "left update")) != CMPS_OK) break;
    if ((status = px.upload(H.ctx->stream)) != CMPS_OK) break;
    if ((status = pl.upload(H.ctx->stream)) != CMPS_OK) break;
    Planar Ucopy = s.U;  // non-owning view
    if ((status = launch_zgemm_fp64(px, false, false, H.LP, Ucopy, X, H.ctx->stream)) != CMPS_OK) break;
    if ((status = launch_zgemm_fp64(pl, true, false, Ucopy, X, out.data, H.ctx->stream)) != CMPS_OK) break;
    if (cudaStreamSynchronize(H.ctx->stream) != cudaSuccess) status = fail(CMPS_ERR_CUDA, "left block update failed");
  } while (false);
  px.release();
  pl.release();
  X.release();
  return status;
}

int right_update(Heff& H, const SvdResult& s, Env& out) {
  const Rules& r = H.rules;
  const ThetaSpace& th = s.th;
  const int nm = (int)th.mq.size();
  const int d = H.d;
  const Bond& A2 = H.R.a;
  Bond nb;
  std::vector<int> sec;
  new_bond(s, nb, sec);
  CMPS_TRY(alloc_env(r, nb, H.D, H.bq, true, out, H.ctx->stream));
  std::set<int> b1s;
  for (auto& kv : H.rp_off) b1s.insert(kv.first[0]);
  GemmPlan py, pr;
  int64_t yt = 0;
  for (int b1 : b1s)
    for (int m = 0; m < nm; ++m) {
      const int64_t k = s.kept[m];
      if (!k) continue;
      int mp = th.find(r.add(th.mq[m], H.bq[b1]));
      if (mp < 0 || !s.kept[mp]) continue;
      // Y^{b1}_m = Vd_m RightPart^{b1}: (k x ncols[m'])
      std::vector<GemmTask> tasks;
      std::vector<GemmTerm> terms;
      for (int s2p = 0; s2p < d; ++s2p) {
        if (th.coloff[mp][s2p] < 0) continue;
        int tp = A2.find(r.add(th.mq[mp], H.sigq[s2p]));
        GemmTask t{};
        t.c_off = th.coloff[mp][s2p];
        t.m = (int32_t)k;
        t.n = (int32_t)A2.sdim[tp];
        t.ldc = (int32_t)th.ncols[mp];
        t.t0 = (int32_t)terms.size();
        for (int s2 = 0; s2 < d; ++s2) {
          if (th.coloff[m][s2] < 0) continue;
          int ta = A2.find(r.add(th.mq[m], H.sigq[s2]));
          auto it = H.rp_off.find({b1, s2, s2p, ta});
          if (it == H.rp_off.end()) continue;
          GemmTerm tm{};
          tm.a_off = s.voff[m] + th.coloff[m][s2];
          tm.lda = (int32_t)th.ncols[m];
          tm.k = (int32_t)A2.sdim[ta];
          tm.b_off = it->second;
          tm.ldb = (int32_t)A2.sdim[tp];
          terms.push_back(tm);
        }
        t.t1 = (int32_t)terms.size();
        tasks.push_back(t);
      }
      if (terms.empty()) continue;
      int64_t yb = yt;
      yt += k * th.ncols[mp];
      int32_t tb = (int32_t)py.terms.size();
      for (auto& tm : terms) py.terms.push_back(tm);
      for (auto& t : tasks) {
        t.c_off += yb;
        t.t0 += tb;
        t.t1 += tb;
        py.tasks.push_back(t);
      }
      // R'^{b1} stored [a, a']: (kept[m] x kept[m']) = Y Vd_{m'}^H
      GemmTask rt{};
      const int ns = nb.nsec();
      rt.c_off = out.off[(size_t)b1 * ns + sec[m]];
      rt.m = (int32_t)k;
      rt.n = (int32_t)s.kept[mp];
      rt.ldc = (int32_t)s.kept[mp];
      rt.t0 = (int32_t)pr.terms.size();
      GemmTerm tm{};
      tm.a_off = yb;
      tm.lda = (int32_t)th.ncols[mp];
      tm.k = (int32_t)th.ncols[mp];
      tm.b_off = s.voff[mp];
      tm.ldb = (int32_t)th.ncols[mp];
      pr.terms.push_back(tm);
      rt.t1 = (int32_t)pr.terms.size();
      pr.tasks.push_back(rt);
    }
  Planar Y;
  CMPS_TRY(Y.alloc(yt));
  int status = CMPS_OK;
  do {
    if ((status = py.validate(false, false, s.Vd.len, H.RP.len, yt, "right update Y")) != CMPS_OK) break;
    if ((status = pr.validate(false, true, yt, s.Vd.len, out.data.len, "right update")) != CMPS_OK) break;
    if ((status = py.upload(H.ctx->stream)) != CMPS_OK) break;
    if ((status = pr.upload(H.ctx->stream)) != CMPS_OK) break;
    Planar Vview = s.Vd;
    if ((status = launch_zgemm_fp64(py, false, false, Vview, H.RP, Y, H.ctx->stream)) != CMPS_OK) break;
    if ((status = launch_zgemm_fp64(pr, false, true, Y, Vview, out.data, H.ctx->stream)) != CMPS_OK) break;
    if (cudaStreamSynchronize(H.ctx->stream) != cudaSuccess) status = fail(CMPS_ERR_CUDA, "right block update failed");
  } while (false);
  py.release();
  pr.release();
  Y.release();
  return status;
}

}  // namespace cmps

struct cmps_svd {
  cmps::SvdResult r;
  ~cmps_svd() {
    r.U.release();
    r.Vd.release();
  }
};


using namespace cmps;

extern "C" {

int cmps_heff_theta_svd(cmps_heff* h, int64_t chi, double max_trunc, cmps_svd** out) {
  if (!h || !h->impl || !out) return fail(CMPS_ERR_ARG, "null argument");
  *out = nullptr;
  if (chi < 0) return fail(CMPS_ERR_ARG, "negative bond dimension");
  CMPS_CUDA(cudaSetDevice(h->impl->device));
  auto* s = new (std::nothrow) cmps_svd();
  if (!s) return fail(CMPS_ERR_NOMEM, "host allocation failed");
  int st = theta_svd(*h->impl, chi, max_trunc, s->r);
  if (st != CMPS_OK) {
    delete s;
    return st;
  }
  *out = s;
  return CMPS_OK;
}

int cmps_svd_destroy(cmps_svd* s) {
  delete s;
  return CMPS_OK;
}

int cmps_svd_info(const cmps_svd* s, int64_t* kept, double* discarded, int64_t* nnz_u, int64_t* nnz_vd) {
  if (!s) return fail(CMPS_ERR_ARG, "null handle");
  const SvdResult& r = s->r;
  if (kept) *kept = (int64_t)r.values.size();
  if (discarded) *discarded = r.discarded;
  // upper bounds: every stored element of the kept factor columns / rows
  int64_t nu = 0, nv = 0;
  for (size_t m = 0; m < r.kept.size(); ++m) {
    nu += r.th.nrows[m] * r.kept[m];
    nv += r.kept[m] * r.th.ncols[m];
  }
  if (nnz_u) *nnz_u = nu;
  if (nnz_vd) *nnz_vd = nv;
  return CMPS_OK;
}

int cmps_svd_routes(const cmps_svd* s, int* n_exact, int* n_gram, int* n_randomized) {
  if (!s) return fail(CMPS_ERR_ARG, "null handle");
  if (n_exact) *n_exact = s->r.routes[0];
  if (n_gram) *n_gram = s->r.routes[1];
  if (n_randomized) *n_randomized = s->r.routes[2];
  return CMPS_OK;
}

int cmps_svd_copy(const cmps_svd* s, double* values, int16_t* new_charges, int64_t* u_colptr, int64_t* u_rowind,
                  double* u_values, int64_t* vd_colptr, int64_t* vd_rowind, double* vd_values) {
  if (!s) return fail(CMPS_ERR_ARG, "null handle");
  const SvdResult& r = s->r;
  const int64_t kept = (int64_t)r.values.size();
  const int nq = r.rules.nq;
  const ThetaSpace& th = r.th;
  const int d = r.d;
  if (values) std::memcpy(values, r.values.data(), sizeof(double) * kept);
  if (new_charges)
    for (int64_t g = 0; g < kept; ++g)
      for (int c = 0; c < nq; ++c) new_charges[g * nq + c] = th.mq[r.order[g].first][c];
  std::vector<double> U(2 * r.U.len), V(2 * r.Vd.len);
  if (r.U.len) CMPS_CUDA(cudaMemcpy(U.data(), r.U.d, sizeof(double) * 2 * r.U.len, cudaMemcpyDeviceToHost));
  if (r.Vd.len) CMPS_CUDA(cudaMemcpy(V.data(), r.Vd.d, sizeof(double) * 2 * r.Vd.len, cudaMemcpyDeviceToHost));
  // U: (d * chiL) x kept, row = s1 + d * a0, column g
  if (u_colptr) {
    int64_t p = 0;
    u_colptr[0] = 0;
    std::vector<std::pair<int64_t, std::pair<double, double>>> col;
    for (int64_t g = 0; g < kept; ++g) {
      const int m = r.order[g].first;
      const int64_t j = r.order[g].second, k = r.kept[m];
      col.clear();
      for (int s1 = 0; s1 < d; ++s1) {
        if (th.rowoff[m][s1] < 0) continue;
        int sa = r.a0.find(r.rules.sub(th.mq[m], r.sigq[s1]));
        for (int64_t q = 0; q < r.a0.sdim[sa]; ++q) {
          int64_t o = r.uoff[m] + (th.rowoff[m][s1] + q) * k + j;
          double re = U[o], im = U[r.U.len + o];
          if (re == 0.0 && im == 0.0) continue;
          col.push_back({s1 + (int64_t)d * r.a0.selem[sa][q], {re, im}});
        }
      }
      std::sort(col.begin(), col.end(), [](auto& a, auto& b) { return a.first < b.first; });
      for (auto& e : col) {
        if (u_rowind) u_rowind[p] = e.first;
        if (u_values) { u_values[2 * p] = e.second.first; u_values[2 * p + 1] = e.second.second; }
        ++p;
      }
      u_colptr[g + 1] = p;
    }
  }
  // V^dagger: kept x (d * chiR), column c = s2 + d * a2
  if (vd_colptr) {
    const int64_t chiR = r.a2.size();
    std::vector<std::vector<std::pair<int64_t, std::pair<double, double>>>> cols(d * chiR);
    for (int m = 0; m < (int)th.mq.size(); ++m) {
      const int64_t k = r.kept[m];
      for (int64_t j = 0; j < k; ++j) {
        const int64_t g = r.gidx[m][j];
        for (int s2 = 0; s2 < d; ++s2) {
          if (th.coloff[m][s2] < 0) continue;
          int t = r.a2.find(r.rules.add(th.mq[m], r.sigq[s2]));
          for (int64_t q = 0; q < r.a2.sdim[t]; ++q) {
            int64_t o = r.voff[m] + j * th.ncols[m] + th.coloff[m][s2] + q;
            double re = V[o], im = V[r.Vd.len + o];
            if (re == 0.0 && im == 0.0) continue;
            cols[s2 + (int64_t)d * r.a2.selem[t][q]].push_back({g, {re, im}});
          }
        }
      }
    }
    int64_t p = 0;
    vd_colptr[0] = 0;
    for (int64_t c = 0; c < d * chiR; ++c) {
      auto& cl = cols[c];
      std::sort(cl.begin(), cl.end(), [](auto& a, auto& b) { return a.first < b.first; });
      for (auto& e : cl) {
        if (vd_rowind) vd_rowind[p] = e.first;
        if (vd_values) { vd_values[2 * p] = e.second.first; vd_values[2 * p + 1] = e.second.second; }
        ++p;
      }
      vd_colptr[c + 1] = p;
    }
  }
  return CMPS_OK;
}

int cmps_heff_left_block(cmps_heff* h, const cmps_svd* s, cmps_block** out) {
  if (!h || !h->impl || !s || !out) return fail(CMPS_ERR_ARG, "null argument");
  *out = nullptr;
  CMPS_CUDA(cudaSetDevice(h->impl->device));
  auto* b = new (std::nothrow) cmps_block();
  if (!b) return fail(CMPS_ERR_NOMEM, "host allocation failed");
  b->rules = h->impl->rules;
  int st = left_update(*h->impl, s->r, b->env);
  if (st != CMPS_OK) { delete b; return st; }
  *out = b;
  return CMPS_OK;
}

int cmps_heff_right_block(cmps_heff* h, const cmps_svd* s, cmps_block** out) {
  if (!h || !h->impl || !s || !out) return fail(CMPS_ERR_ARG, "null argument");
  *out = nullptr;
  CMPS_CUDA(cudaSetDevice(h->impl->device));
  auto* b = new (std::nothrow) cmps_block();
  if (!b) return fail(CMPS_ERR_NOMEM, "host allocation failed");
  b->rules = h->impl->rules;
  int st = right_update(*h->impl, s->r, b->env);
  if (st != CMPS_OK) { delete b; return st; }
  *out = b;
  return CMPS_OK;
}

int cmps_block_destroy(cmps_block* b) {
  delete b;
  return CMPS_OK;
}

int cmps_block_info(const cmps_block* b, int64_t* chi, int64_t* mpo_dim, int64_t* nnz) {
  if (!b) return fail(CMPS_ERR_ARG, "null handle");
  if (chi) *chi = b->env.a.size();
  if (mpo_dim) *mpo_dim = b->env.D;
  if (nnz) *nnz = b->env.data.len;  // upper bound
  return CMPS_OK;
}

int cmps_block_copy(const cmps_block* b, int16_t* a_charges, int64_t* colptr, int64_t* rowind, double* values) {
  if (!b) return fail(CMPS_ERR_ARG, "null handle");
  const Env& e = b->env;
  const int nq = b->rules.nq;
  const int64_t chi = e.a.size();
  if (a_charges)
    for (int64_t i = 0; i < chi; ++i)
      for (int c = 0; c < nq; ++c) a_charges[i * nq + c] = e.a.sq[e.a.esec[i]][c];
  if (!colptr) return CMPS_OK;
  std::vector<double> h(2 * e.data.len);
  if (e.data.len) CMPS_CUDA(cudaMemcpy(h.data(), e.data.d, sizeof(double) * 2 * e.data.len, cudaMemcpyDeviceToHost));
  // matrix rows a', cols b + D * a
  const int ns = e.a.nsec();
  int64_t p = 0;
  colptr[0] = 0;
  std::vector<std::pair<int64_t, std::pair<double, double>>> col;
  for (int64_t a = 0; a < chi; ++a) {
    const int s = e.a.esec[a];
    const int64_t pa = e.a.epos[a];
    for (int bb = 0; bb < e.D; ++bb) {
      col.clear();
      int64_t o = e.off[(size_t)bb * ns + s];
      if (o >= 0) {
        int sp = e.partner[(size_t)bb * ns + s];
        for (int64_t q = 0; q < e.a.sdim[sp]; ++q) {
          int64_t ap = e.a.selem[sp][q];
          int64_t idx = e.right ? o + pa * e.a.sdim[sp] + q : o + q * e.a.sdim[s] + pa;
          double re = h[idx], im = h[e.data.len + idx];
          if (re == 0.0 && im == 0.0) continue;
          col.push_back({ap, {re, im}});
        }
        std::sort(col.begin(), col.end(), [](auto& x, auto& y) { return x.first < y.first; });
      }
      for (auto& v : col) {
        if (rowind) rowind[p] = v.first;
        if (values) { values[2 * p] = v.second.first; values[2 * p + 1] = v.second.second; }
        ++p;
      }
      colptr[bb + (int64_t)e.D * a + 1] = p;
    }
  }
  return CMPS_OK;
}

}  // extern "C"
