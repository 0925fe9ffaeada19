// The iDMRG unit cell of the last growth step, its orthogonalisation and the
// energy per vertex: what the iDMRG driver measures after every step
// (iDMRG_DRV.cpp:71-77: Orthogonalise, then iTwoVertexEnergy).
//
// The cell (UnitCell(MPSDecomposition, PreviousLambda), UnitCell.hpp:42-47)
// is A0[s1] = U[s1] and A1[s2] = diag(s) V^dagger[s2] diag(1/lambda_prev),
// its right bond identified element by element with its left bond.  With
// M[s1,s2] = A0[s1] A1[s2], the left transfer map is L(l) = sum M^dag l M
// (l indexed [bra, ket]) and the right map R(r) = sum M r M^dag (r indexed
// [ket, bra]); LeftED / RightED (measurement.cpp:456-575) are their
// dominant eigenpairs, made Hermitian.  Orthogonalise (measurement.cpp:
// 180-246) factors them (SqrtDR, MPX_matrix.cpp:829-911: l = X^dag X with
// eigenvalues |w| <= 100 eps max|w| dropped, mixed signs a failure), takes
// the new boundary values Lambda' from the SVD of X Y (r = Y Y^dag) and
// regauges the cell; iTwoVertexEnergy (measurement.cpp:371-397) then traces
// the on-vertex term H1 = W[D-1, 0] of both sites, the bond
// sum_k RowX_k ColX_k (RowX_k = W[D-1, k], ColX_k = W[k, 0]) inside the cell
// and the bond into the next cell against Lambda'^2.
//
// The dominant eigenpairs are found on charge blocks: the maps preserve the
// charge difference of their two indices and start from the identity, so the
// fixed points stay block diagonal in the bond's charge sectors.  Each map is
// four grouped FP64 GEMM launches over the sector blocks of U and of
// diag(s) V^dagger diag(1/lambda_prev), at O(sum of sector dim^3) instead of
// O(chi^3) per application; the converged blocks are then placed in dense
// chi0 x chi0 matrices for the rest of the measurement.
//
// Here the same numbers come from the fixed points directly, which the
// regauging leaves invariant: <O> = Tr[T_O(l) r] / (eta Tr[l r]) for an
// operator on one cell (T_O the left map with O inserted) and
// Tr[T_O2(T_O1(l)) r] / (eta^2 Tr[l r]) for the bond between two cells;
// Lambda'^2 are the eigenvalues of X r X^dag, normalised.  All operators act
// on the dense cell: cuBLAS ZGEMMs on the column-major A0[s] (chi0 x chi1)
// and A1[s] (chi1 x chi0).  The dominant eigenpairs come from a restarted
// Arnoldi iteration on chi0 x chi0 matrices with two classical Gram-Schmidt
// passes; its small Hessenberg eigenproblem is solved on the host (power
// iteration, then inverse iteration at the Rayleigh quotient).
#include <cublas_v2.h>
#include <cuComplex.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <functional>
#include <map>
#include <vector>

#include "heff.h"

namespace cmps {

namespace {

using cplx = cuDoubleComplex;
using zc = std::complex<double>;
constexpr double kEps = 2.220446049250313e-16;

int grid_of(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 32)); }

// Scatter one row-major planar block into a stack of column-major matrices:
// entry (r, c) lands in matrix sig (from the row map, or from the column map
// when rsig is null) at (rdst[r], cdst[c]), scaled by rscale[r] * cscale[c].
__global__ void k_scatter_cell(const double* __restrict__ re, const double* __restrict__ im, int64_t nr, int64_t nc,
                               const int32_t* __restrict__ rsig, const int32_t* __restrict__ csig,
                               const int64_t* __restrict__ rdst, const int64_t* __restrict__ cdst,
                               const double* __restrict__ rscale, const double* __restrict__ cscale,
                               cplx* __restrict__ dst, int64_t ld, int64_t stride) {
  const int64_t n = nr * nc;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e / nc, c = e % nc;
    const int64_t sig = rsig ? rsig[r] : csig[c];
    const double f = (rscale ? rscale[r] : 1.0) * (cscale ? cscale[c] : 1.0);
    dst[sig * stride + rdst[r] + ld * cdst[c]] = make_cuDoubleComplex(re[e] * f, im[e] * f);
  }
}

// interleaved complex <-> two planes
__global__ void k_deinterleave(const cplx* __restrict__ in, int64_t n, double* __restrict__ re,
                               double* __restrict__ im) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    re[e] = in[e].x;
    im[e] = in[e].y;
  }
}
__global__ void k_interleave(const double* __restrict__ re, const double* __restrict__ im, int64_t n,
                             cplx* __restrict__ out) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
    out[e] = make_cuDoubleComplex(re[e], im[e]);
}
// out[r, c] = rs[r] * in[r, c] * cs[c], one row-major block (planar)
__global__ void k_scale_rc(const double* __restrict__ re, const double* __restrict__ im, int64_t rows, int64_t cols,
                           const double* __restrict__ rs, const double* __restrict__ cs, double* __restrict__ ore,
                           double* __restrict__ oim) {
  const int64_t n = rows * cols;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const double f = rs[e / cols] * cs[e % cols];
    ore[e] = re[e] * f;
    oim[e] = im[e] * f;
  }
}
// dense[dst[e]] = v[e]
__global__ void k_scatter_index(const cplx* __restrict__ v, const int64_t* __restrict__ dst, int64_t n,
                                cplx* __restrict__ dense) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
    dense[dst[e]] = v[e];
}

// v <- Hermitian part of (phase * v), in place (n x n, column-major).
__global__ void k_hermitize(cplx* __restrict__ v, int64_t n, cplx phase) {
  const int64_t tot = n * n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e % n, j = e / n;
    if (i > j) continue;
    const cplx a = cuCmul(phase, v[i + n * j]);
    const cplx b = cuCmul(phase, v[j + n * i]);
    const cplx h = make_cuDoubleComplex(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
    v[i + n * j] = h;
    v[j + n * i] = cuConj(h);
  }
}

// out (m x m) = in (m x m) transposed, for `count` matrices of stride m*m.
__global__ void k_transpose_stack(const cplx* __restrict__ in, cplx* __restrict__ out, int64_t m, int64_t count) {
  const int64_t tot = m * m * count;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t q = e / (m * m), w = e % (m * m), i = w % m, j = w / m;
    out[q * m * m + j + m * i] = in[e];
  }
}

// X[k, j] = root[k] * conj(E[j, keep[k]]): (kL x n), column-major.
__global__ void k_make_x(const cplx* __restrict__ E, int64_t n, const int32_t* __restrict__ keep,
                         const double* __restrict__ root, int64_t kl, cplx* __restrict__ X) {
  const int64_t tot = kl * n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = e % kl, j = e / kl;
    const cplx v = E[j + n * keep[k]];
    X[e] = make_cuDoubleComplex(root[k] * v.x, -root[k] * v.y);
  }
}

struct Cell {
  int d = 0;
  int64_t c0 = 0, c1 = 0;
  cplx* A0 = nullptr;  // d x (c0 x c1)
  cplx* A1 = nullptr;  // d x (c1 x c0)
  cplx* a0(int s) const { return A0 + (int64_t)s * c0 * c1; }
  cplx* a1(int s) const { return A1 + (int64_t)s * c1 * c0; }
};

struct Blas {
  cublasHandle_t h;
  int st = CMPS_OK;
  void gemm(cublasOperation_t ta, cublasOperation_t tb, int64_t m, int64_t n, int64_t k, cplx alpha, const cplx* A,
            int64_t lda, const cplx* B, int64_t ldb, cplx beta, cplx* C, int64_t ldc) {
    if (st != CMPS_OK) return;
    if (cublasZgemm(h, ta, tb, (int)m, (int)n, (int)k, &alpha, A, (int)lda, B, (int)ldb, &beta, C, (int)ldc) !=
        CUBLAS_STATUS_SUCCESS)
      st = fail(CMPS_ERR_CUDA, "unit cell: cublasZgemm failed");
  }
};

const cplx kOne = {1.0, 0.0}, kZero = {0.0, 0.0};

// The left and right transfer maps on block-diagonal fixed points.  A vector
// is the concatenation of the row-major blocks l_s (dim s x dim s) over the
// sectors s of the cell's end bond.  Left: X = l_s A0, W_m = sum A0^H X,
// Y = W_m A1, l'_u = sum A1^H Y; right: Z = A1 r_u, V_m = sum Z A1^H,
// P = A0 V_m, r'_s = sum P A0^H -- A0[s1] the rows of U's block m of state
// s1 (sector s = m - q(s1)), A1[s2] the columns of the scaled V^dagger's
// block m of state s2 (sector u = m + q(s2)).
struct BlockMaps {
  int64_t nb = 0;
  std::vector<int64_t> boff, bdim;  // per bond sector
  std::vector<int64_t> dense_of;    // vector entry -> column-major dense index
  GemmPlan L1, L2, L3, L4, R1, R2, R3, R4;
  Planar vin, vout, X, W, Y, Vs;
  const Planar* U = nullptr;
  void release() {
    for (GemmPlan* p : {&L1, &L2, &L3, &L4, &R1, &R2, &R3, &R4}) p->release();
    for (Planar* q : {&vin, &vout, &X, &W, &Y, &Vs}) q->release();
  }
};

int build_block_maps(const SvdResult& S, const std::vector<double>& lam, const std::vector<double>& inv_prev,
                     cudaStream_t st, BlockMaps& M) {
  const ThetaSpace& th = S.th;
  const Bond& A0 = S.a0;
  const Bond& A2 = S.a2;
  const int nm = (int)th.mq.size(), d = S.d, ns = A0.nsec();
  const int64_t c0 = A0.size();
  M.U = &S.U;
  M.boff.assign(ns, 0);
  M.bdim.assign(ns, 0);
  M.dense_of.clear();
  for (int s = 0; s < ns; ++s) {
    M.boff[s] = M.nb;
    M.bdim[s] = A0.sdim[s];
    for (int64_t p = 0; p < A0.sdim[s]; ++p)
      for (int64_t q = 0; q < A0.sdim[s]; ++q) M.dense_of.push_back(A0.selem[s][p] + c0 * A0.selem[s][q]);
    M.nb += A0.sdim[s] * A0.sdim[s];
  }
  // a2 sector -> the a0 sector of the same charge (the cell's end bonds are identified)
  auto a0_of_a2 = [&](int t) { return A0.find(A2.sq[t]); };
  std::map<std::pair<int, int>, int64_t> xo, yo;  // (state, m) -> offset
  std::vector<int64_t> wo(nm, -1);
  int64_t xl = 0, wl = 0, yl = 0;
  for (int m = 0; m < nm; ++m) {
    const int64_t k = S.kept[m];
    if (!k) continue;
    wo[m] = wl;
    wl += k * k;
    for (int s1 = 0; s1 < d; ++s1) {
      if (th.rowoff[m][s1] < 0) continue;
      const int sa = A0.find(S.rules.sub(th.mq[m], S.sigq[s1]));
      if (sa < 0) return fail(CMPS_ERR_STATE, "unit cell: left tensor sector");
      xo[{s1, m}] = xl;
      xl += A0.sdim[sa] * k;
    }
    for (int s2 = 0; s2 < d; ++s2) {
      if (th.coloff[m][s2] < 0) continue;
      const int t = A2.find(S.rules.add(th.mq[m], S.sigq[s2]));
      if (t < 0 || a0_of_a2(t) < 0 || A0.sdim[a0_of_a2(t)] != A2.sdim[t])
        return fail(CMPS_ERR_STATE, "unit cell: end bonds differ");
      yo[{s2, m}] = yl;
      yl += k * A2.sdim[t];
    }
  }
  CMPS_TRY(M.vin.alloc(std::max<int64_t>(1, M.nb)));
  CMPS_TRY(M.vout.alloc(std::max<int64_t>(1, M.nb)));
  CMPS_TRY(M.X.alloc(std::max<int64_t>(1, xl)));
  CMPS_TRY(M.W.alloc(std::max<int64_t>(1, wl)));
  CMPS_TRY(M.Y.alloc(std::max<int64_t>(1, yl)));
  CMPS_TRY(M.Vs.alloc(std::max<int64_t>(1, S.Vd.len)));
  // A1 = diag(s) V^dagger diag(1 / lambda_prev), block by block
  for (int m = 0; m < nm; ++m) {
    const int64_t k = S.kept[m], C = th.ncols[m];
    if (!k) continue;
    std::vector<double> rs(k), cs(C, 0.0);
    for (int64_t j = 0; j < k; ++j) rs[j] = lam[S.gidx[m][j]];
    for (int s2 = 0; s2 < d; ++s2) {
      if (th.coloff[m][s2] < 0) continue;
      const int t = A2.find(S.rules.add(th.mq[m], S.sigq[s2]));
      for (int64_t p = 0; p < A2.sdim[t]; ++p) cs[th.coloff[m][s2] + p] = inv_prev[A2.selem[t][p]];
    }
    double *d_rs = nullptr, *d_cs = nullptr;
    if (dmalloc(&d_rs, sizeof(double) * k) != cudaSuccess || dmalloc(&d_cs, sizeof(double) * C) != cudaSuccess) {
      if (d_rs) dfree(d_rs);
      return fail(CMPS_ERR_NOMEM, "unit cell: scale allocation failed");
    }
    int rc = copy_wait(d_rs, rs.data(), sizeof(double) * k, cudaMemcpyHostToDevice, st);
    if (rc == CMPS_OK) rc = copy_wait(d_cs, cs.data(), sizeof(double) * C, cudaMemcpyHostToDevice, st);
    if (rc == CMPS_OK) {
      k_scale_rc<<<grid_of(k * C), 256, 0, st>>>(S.Vd.re() + S.voff[m], S.Vd.im() + S.voff[m], k, C, d_rs, d_cs,
                                                 M.Vs.re() + S.voff[m], M.Vs.im() + S.voff[m]);
      if (cudaStreamSynchronize(st) != cudaSuccess) rc = fail(CMPS_ERR_CUDA, "unit cell: scaling failed");
    }
    dfree(d_rs);
    dfree(d_cs);
    CMPS_TRY(rc);
  }
  auto task = [](GemmPlan& p, int64_t c_off, int64_t m, int64_t n, int64_t ldc) {
    GemmTask t{};
    t.c_off = c_off;
    t.m = (int32_t)m;
    t.n = (int32_t)n;
    t.ldc = (int32_t)ldc;
    t.t0 = t.t1 = (int32_t)p.terms.size();
    p.tasks.push_back(t);
  };
  auto term = [](GemmPlan& p, int64_t a_off, int64_t lda, int64_t b_off, int64_t ldb, int64_t k) {
    GemmTerm tm{};
    tm.a_off = a_off;
    tm.lda = (int32_t)lda;
    tm.b_off = b_off;
    tm.ldb = (int32_t)ldb;
    tm.k = (int32_t)k;
    p.terms.push_back(tm);
    p.tasks.back().t1 = (int32_t)p.terms.size();
  };
  // per (state, m): the A0 block (rows of state s1: dim sa x k, ld k) and
  // the A1 block (columns of state s2: k x dim t, ld ncols)
  for (int m = 0; m < nm; ++m) {
    const int64_t k = S.kept[m], C = th.ncols[m];
    if (!k) continue;
    for (int s1 = 0; s1 < d; ++s1) {
      if (th.rowoff[m][s1] < 0) continue;
      const int sa = A0.find(S.rules.sub(th.mq[m], S.sigq[s1]));
      const int64_t ds = A0.sdim[sa], a0b = S.uoff[m] + th.rowoff[m][s1] * k, x = xo[{s1, m}];
      task(M.L1, x, ds, k, k);                       // X = l_s A0
      term(M.L1, M.boff[sa], ds, a0b, k, ds);
      task(M.R3, x, ds, k, k);                       // P = A0 V_m
      term(M.R3, a0b, k, wo[m], k, k);
    }
    task(M.L2, wo[m], k, k, k);                      // W_m = sum A0^H X
    for (int s1 = 0; s1 < d; ++s1) {
      if (th.rowoff[m][s1] < 0) continue;
      const int sa = A0.find(S.rules.sub(th.mq[m], S.sigq[s1]));
      term(M.L2, S.uoff[m] + th.rowoff[m][s1] * k, k, xo[{s1, m}], k, A0.sdim[sa]);
    }
    task(M.R2, wo[m], k, k, k);                      // V_m = sum Z A1^H
    for (int s2 = 0; s2 < d; ++s2) {
      if (th.coloff[m][s2] < 0) continue;
      const int t = A2.find(S.rules.add(th.mq[m], S.sigq[s2]));
      const int64_t du = A2.sdim[t], a1b = S.voff[m] + th.coloff[m][s2], y = yo[{s2, m}];
      term(M.R2, y, du, a1b, C, du);
      task(M.L3, y, k, du, du);                      // Y = W_m A1
      term(M.L3, wo[m], k, a1b, C, k);
      task(M.R1, y, k, du, du);                      // Z = A1 r_u
      term(M.R1, a1b, C, M.boff[a0_of_a2(t)], du, du);
    }
  }
  for (int sb = 0; sb < ns; ++sb) {
    const int64_t db = A0.sdim[sb];
    task(M.L4, M.boff[sb], db, db, db);              // l'_u = sum A1^H Y
    task(M.R4, M.boff[sb], db, db, db);              // r'_s = sum P A0^H
  }
  // L4 / R4: one task per output sector, its terms from every (state, m) that reaches it
  {
    std::vector<std::vector<GemmTerm>> l4(ns), r4(ns);
    for (int m = 0; m < nm; ++m) {
      const int64_t k = S.kept[m], C = th.ncols[m];
      if (!k) continue;
      for (int s2 = 0; s2 < d; ++s2) {
        if (th.coloff[m][s2] < 0) continue;
        const int t = A2.find(S.rules.add(th.mq[m], S.sigq[s2]));
        GemmTerm tm{};
        tm.a_off = S.voff[m] + th.coloff[m][s2];
        tm.lda = (int32_t)C;
        tm.b_off = yo[{s2, m}];
        tm.ldb = (int32_t)A2.sdim[t];
        tm.k = (int32_t)k;
        l4[a0_of_a2(t)].push_back(tm);
      }
      for (int s1 = 0; s1 < d; ++s1) {
        if (th.rowoff[m][s1] < 0) continue;
        const int sa = A0.find(S.rules.sub(th.mq[m], S.sigq[s1]));
        GemmTerm tm{};
        tm.a_off = xo[{s1, m}];
        tm.lda = (int32_t)k;
        tm.b_off = S.uoff[m] + th.rowoff[m][s1] * k;
        tm.ldb = (int32_t)k;
        tm.k = (int32_t)k;
        r4[sa].push_back(tm);
      }
    }
    for (int pass = 0; pass < 2; ++pass) {
      GemmPlan& p = pass == 0 ? M.L4 : M.R4;
      std::vector<std::vector<GemmTerm>>& lists = pass == 0 ? l4 : r4;
      p.terms.clear();
      for (int sb = 0; sb < ns; ++sb) {
        p.tasks[sb].t0 = (int32_t)p.terms.size();
        p.terms.insert(p.terms.end(), lists[sb].begin(), lists[sb].end());
        p.tasks[sb].t1 = (int32_t)p.terms.size();
      }
    }
  }
  // every operand and output range inside its buffer, then upload
  const int64_t ul = S.U.len, vl = M.Vs.len, nb = std::max<int64_t>(1, M.nb);
  struct Check {
    GemmPlan* p;
    bool ah, bh;
    int64_t a, b, c;
    const char* what;
  };
  const Check checks[] = {{&M.L1, false, false, nb, ul, M.X.len, "unit cell L1"},
                          {&M.L2, true, false, ul, M.X.len, M.W.len, "unit cell L2"},
                          {&M.L3, false, false, M.W.len, vl, M.Y.len, "unit cell L3"},
                          {&M.L4, true, false, vl, M.Y.len, nb, "unit cell L4"},
                          {&M.R1, false, false, vl, nb, M.Y.len, "unit cell R1"},
                          {&M.R2, false, true, M.Y.len, vl, M.W.len, "unit cell R2"},
                          {&M.R3, false, false, ul, M.W.len, M.X.len, "unit cell R3"},
                          {&M.R4, false, true, M.X.len, ul, nb, "unit cell R4"}};
  for (const Check& c : checks) {
    CMPS_TRY(c.p->validate(c.ah, c.bh, c.a, c.b, c.c, c.what));
    CMPS_TRY(c.p->upload(st));
  }
  return CMPS_OK;
}

// out = L(in) or R(in) on block vectors (interleaved, nb entries)
int apply_block_map(BlockMaps& M, bool left, const cplx* in, cplx* out, cudaStream_t st) {
  const int64_t nb = M.nb;
  k_deinterleave<<<grid_of(nb), 256, 0, st>>>(in, nb, M.vin.re(), M.vin.im());
  CMPS_CUDA(cudaMemsetAsync(M.vout.d, 0, sizeof(double) * 2 * M.vout.len, st));
  if (left) {
    CMPS_TRY(launch_zgemm_fp64(M.L1, false, false, M.vin, *M.U, M.X, st));
    CMPS_TRY(launch_zgemm_fp64(M.L2, true, false, *M.U, M.X, M.W, st));
    CMPS_TRY(launch_zgemm_fp64(M.L3, false, false, M.W, M.Vs, M.Y, st));
    CMPS_TRY(launch_zgemm_fp64(M.L4, true, false, M.Vs, M.Y, M.vout, st));
  } else {
    CMPS_TRY(launch_zgemm_fp64(M.R1, false, false, M.Vs, M.vin, M.Y, st));
    CMPS_TRY(launch_zgemm_fp64(M.R2, false, true, M.Y, M.Vs, M.W, st));
    CMPS_TRY(launch_zgemm_fp64(M.R3, false, false, *M.U, M.W, M.X, st));
    CMPS_TRY(launch_zgemm_fp64(M.R4, false, true, M.X, *M.U, M.vout, st));
  }
  k_interleave<<<grid_of(nb), 256, 0, st>>>(M.vout.re(), M.vout.im(), nb, out);
  CMPS_CUDA(cudaGetLastError());
  return CMPS_OK;
}

// Dominant eigenpair of a small complex matrix H (k x k, column-major):
// power iteration from a fixed start, then inverse iteration at the
// Rayleigh quotient.  Returns false when no iterate is finite.
bool small_dominant(int k, const std::vector<zc>& H, zc* theta, std::vector<zc>& y) {
  auto mul = [&](const std::vector<zc>& x) {
    std::vector<zc> o(k, 0.0);
    for (int j = 0; j < k; ++j)
      for (int i = 0; i < k; ++i) o[i] += H[i + (size_t)k * j] * x[j];
    return o;
  };
  auto normalise = [&](std::vector<zc>& x) {
    double s = 0.0;
    for (auto& v : x) s += std::norm(v);
    s = std::sqrt(s);
    if (!(s > 0.0) || !std::isfinite(s)) return false;
    for (auto& v : x) v /= s;
    return true;
  };
  auto rayleigh = [&](const std::vector<zc>& x) {
    const std::vector<zc> hx = mul(x);
    zc num = 0.0;
    for (int i = 0; i < k; ++i) num += std::conj(x[i]) * hx[i];
    return num;
  };
  y.assign(k, zc(1.0, 0.0));
  for (int i = 0; i < k; ++i) y[i] = zc(1.0 + 0.01 * i, 0.0);
  if (!normalise(y)) return false;
  for (int it = 0; it < 400; ++it) {
    y = mul(y);
    if (!normalise(y)) return false;
  }
  zc mu = rayleigh(y);
  for (int it = 0; it < 4; ++it) {
    // solve (H - mu I) z = y by Gaussian elimination with partial pivoting
    std::vector<zc> A(H);
    const zc shift = mu + zc(1e-13 * std::max(1.0, std::abs(mu)), 0.0);
    for (int i = 0; i < k; ++i) A[i + (size_t)k * i] -= shift;
    std::vector<zc> z(y);
    bool ok = true;
    for (int col = 0; col < k && ok; ++col) {
      int p = col;
      for (int r = col + 1; r < k; ++r)
        if (std::abs(A[r + (size_t)k * col]) > std::abs(A[p + (size_t)k * col])) p = r;
      if (std::abs(A[p + (size_t)k * col]) == 0.0) {
        ok = false;
        break;
      }
      if (p != col) {
        for (int j = 0; j < k; ++j) std::swap(A[col + (size_t)k * j], A[p + (size_t)k * j]);
        std::swap(z[col], z[p]);
      }
      for (int r = col + 1; r < k; ++r) {
        const zc f = A[r + (size_t)k * col] / A[col + (size_t)k * col];
        if (f == zc(0.0)) continue;
        for (int j = col; j < k; ++j) A[r + (size_t)k * j] -= f * A[col + (size_t)k * j];
        z[r] -= f * z[col];
      }
    }
    if (!ok) break;
    for (int r = k - 1; r >= 0; --r) {
      zc s = z[r];
      for (int j = r + 1; j < k; ++j) s -= A[r + (size_t)k * j] * z[j];
      z[r] = s / A[r + (size_t)k * r];
    }
    if (!normalise(z)) break;
    y = z;
    mu = rayleigh(y);
  }
  *theta = rayleigh(y);
  return std::isfinite(theta->real()) && std::isfinite(theta->imag());
}

// Dominant eigenpair of a map (apply: out = map(in), n entries) by restarted
// Arnoldi; x holds the start vector and receives the eigenvector.  V:
// (kdim + 1) x n workspace.
int dominant(Blas& b, cudaStream_t st, int64_t n, const std::function<int(const cplx*, cplx*)>& apply, double tol,
             int kdim, int max_restarts, cplx* x, cplx* V, cplx* hvec, zc* eta) {
  kdim = std::max(2, std::min<int>(kdim, (int)std::min<int64_t>(n, 64)));
  zc theta = 0.0;
  bool converged = false;
  for (int restart = 0; restart < std::max(1, max_restarts) && !converged; ++restart) {
    double nrm = 0.0;
    if (cublasDznrm2(b.h, (int)n, x, 1, &nrm) != CUBLAS_STATUS_SUCCESS || !(nrm > 0.0))
      return fail(CMPS_ERR_SOLVER, "unit cell: zero Arnoldi start vector");
    const double inv = 1.0 / nrm;
    cudaMemcpyAsync(V, x, sizeof(cplx) * n, cudaMemcpyDeviceToDevice, st);
    cublasZdscal(b.h, (int)n, &inv, V, 1);
    std::vector<zc> H((size_t)(kdim + 1) * kdim, 0.0);  // column-major (kdim+1) x kdim
    std::vector<zc> y;
    int k = 0;
    for (int j = 0; j < kdim; ++j) {
      cplx* vj = V + (int64_t)j * n;
      cplx* w = V + (int64_t)(j + 1) * n;
      CMPS_TRY(apply(vj, w));
      if (b.st != CMPS_OK) return b.st;
      for (int pass = 0; pass < 2; ++pass) {
        const cplx mone = {-1.0, 0.0};
        if (cublasZgemv(b.h, CUBLAS_OP_C, (int)n, j + 1, &kOne, V, (int)n, w, 1, &kZero, hvec, 1) !=
                CUBLAS_STATUS_SUCCESS ||
            cublasZgemv(b.h, CUBLAS_OP_N, (int)n, j + 1, &mone, V, (int)n, hvec, 1, &kOne, w, 1) !=
                CUBLAS_STATUS_SUCCESS)
          return fail(CMPS_ERR_CUDA, "unit cell: Gram-Schmidt failed");
        std::vector<cplx> hh(j + 1);
        cudaMemcpyAsync(hh.data(), hvec, sizeof(cplx) * (j + 1), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) return fail(CMPS_ERR_CUDA, "unit cell: Arnoldi step failed");
        for (int i = 0; i <= j; ++i) H[i + (size_t)(kdim + 1) * j] += zc(hh[i].x, hh[i].y);
      }
      double beta = 0.0;
      cublasDznrm2(b.h, (int)n, w, 1, &beta);
      H[(j + 1) + (size_t)(kdim + 1) * j] = beta;
      k = j + 1;
      std::vector<zc> Hk((size_t)k * k);
      for (int jj = 0; jj < k; ++jj)
        for (int ii = 0; ii < k; ++ii) Hk[ii + (size_t)k * jj] = H[ii + (size_t)(kdim + 1) * jj];
      if (!small_dominant(k, Hk, &theta, y)) return fail(CMPS_ERR_SOLVER, "unit cell: Hessenberg eigenproblem failed");
      const double resid = beta * std::abs(y[k - 1]);
      if (resid <= tol * std::abs(theta) || !(beta > 1e-300)) {
        converged = true;
        break;
      }
      if (j + 1 < kdim) {
        const double ib = 1.0 / beta;
        cublasZdscal(b.h, (int)n, &ib, w, 1);
      }
    }
    // Ritz vector x = V_k y
    std::vector<cplx> yc(k);
    for (int i = 0; i < k; ++i) yc[i] = make_cuDoubleComplex(y[i].real(), y[i].imag());
    cudaMemcpyAsync(hvec, yc.data(), sizeof(cplx) * k, cudaMemcpyHostToDevice, st);
    if (cublasZgemv(b.h, CUBLAS_OP_N, (int)n, k, &kOne, V, (int)n, hvec, 1, &kZero, x, 1) != CUBLAS_STATUS_SUCCESS)
      return fail(CMPS_ERR_CUDA, "unit cell: Ritz vector failed");
    if (cudaStreamSynchronize(st) != cudaSuccess) return fail(CMPS_ERR_CUDA, "unit cell: Ritz vector failed");
  }
  if (!converged) return fail(CMPS_ERR_SOLVER, "unit cell: transfer-matrix eigensolver did not converge");
  *eta = theta;
  return CMPS_OK;
}

// trace of a column-major n x n matrix, on the host
zc trace_of(const cplx* dA, int64_t n, cudaStream_t st) {
  std::vector<cplx> h((size_t)n * n);
  cudaMemcpyAsync(h.data(), dA, sizeof(cplx) * n * n, cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  zc t = 0.0;
  for (int64_t i = 0; i < n; ++i) t += zc(h[i + n * i].x, h[i + n * i].y);
  return t;
}

}  // namespace

int unit_cell_measure(cmps_context* ctx, const SvdResult& S, const std::vector<double>& lam,
                      const std::vector<double>& lam_prev, const std::vector<WEntry>& W, int D, double tol, int kdim,
                      UnitCellMeasure* out) {
  cudaStream_t st = ctx->stream;
  const int d = S.d;
  const int64_t c0 = S.a0.size(), c1 = (int64_t)S.values.size();
  if (S.a0.element_charges() != S.a2.element_charges() || (int64_t)lam_prev.size() != c0 ||
      (int64_t)lam.size() != c1 || c0 < 1 || c1 < 1)
    return fail(CMPS_ERR_STATE, "unit cell: the step's end bonds differ (no previous step to pair them)");
  if (D < 3) return fail(CMPS_ERR_STATE, "unit cell: MPO bond dimension below 3");
  const ThetaSpace& th = S.th;
  const int nm = (int)th.mq.size();
  void* blas_v = nullptr;
  void* sol_v = nullptr;
  CMPS_TRY(context_blas(ctx, &blas_v));
  CMPS_TRY(context_solver(ctx, &sol_v));
  Blas bl{(cublasHandle_t)blas_v};
  cusolverDnHandle_t sol = (cusolverDnHandle_t)sol_v;

  std::vector<void*> allocs;
  auto alloc = [&](auto** p, size_t bytes) -> int {
    if (dmalloc((void**)p, std::max<size_t>(bytes, 16)) != cudaSuccess)
      return fail(CMPS_ERR_NOMEM, "unit cell: device allocation failed");
    allocs.push_back((void*)*p);
    return CMPS_OK;
  };
  struct Free {
    std::vector<void*>& a;
    ~Free() {
      for (void* p : a) dfree(p);
    }
  } free_guard{allocs};

  // ---- dense cell ----
  Cell c{d, c0, c1, nullptr, nullptr};
  CMPS_TRY(alloc(&c.A0, sizeof(cplx) * d * c0 * c1));
  CMPS_TRY(alloc(&c.A1, sizeof(cplx) * d * c1 * c0));
  CMPS_CUDA(cudaMemsetAsync(c.A0, 0, sizeof(cplx) * d * c0 * c1, st));
  CMPS_CUDA(cudaMemsetAsync(c.A1, 0, sizeof(cplx) * d * c1 * c0, st));
  std::vector<double> inv_prev(c0);
  for (int64_t j = 0; j < c0; ++j) inv_prev[j] = lam_prev[j] != 0.0 ? 1.0 / lam_prev[j] : 0.0;
  for (int m = 0; m < nm; ++m) {
    const int64_t k = S.kept[m];
    if (!k) continue;
    const int64_t R = th.nrows[m], C = th.ncols[m];
    std::vector<int32_t> rsig(R, -1), csig(C, -1);
    std::vector<int64_t> rdst(R, -1), cdst_c(C, -1), kcol(k);
    std::vector<double> kscale(k), cscale(C, 0.0);
    for (int s1 = 0; s1 < d; ++s1) {
      if (th.rowoff[m][s1] < 0) continue;
      const int sa = S.a0.find(S.rules.sub(th.mq[m], S.sigq[s1]));
      for (int64_t p = 0; p < S.a0.sdim[sa]; ++p) {
        rsig[th.rowoff[m][s1] + p] = s1;
        rdst[th.rowoff[m][s1] + p] = S.a0.selem[sa][p];
      }
    }
    for (int s2 = 0; s2 < d; ++s2) {
      if (th.coloff[m][s2] < 0) continue;
      const int t = S.a2.find(S.rules.add(th.mq[m], S.sigq[s2]));
      for (int64_t p = 0; p < S.a2.sdim[t]; ++p) {
        const int64_t j = S.a2.selem[t][p];
        csig[th.coloff[m][s2] + p] = s2;
        cdst_c[th.coloff[m][s2] + p] = j;
        cscale[th.coloff[m][s2] + p] = inv_prev[j];
      }
    }
    for (int64_t j = 0; j < k; ++j) {
      kcol[j] = S.gidx[m][j];
      kscale[j] = lam[S.gidx[m][j]];
    }
    for (int64_t r = 0; r < R; ++r)
      if (rsig[r] < 0 || rdst[r] < 0 || rdst[r] >= c0) return fail(CMPS_ERR_STATE, "unit cell: row map");
    for (int64_t q = 0; q < C; ++q)
      if (csig[q] < 0 || cdst_c[q] < 0 || cdst_c[q] >= c0) return fail(CMPS_ERR_STATE, "unit cell: column map");
    for (int64_t j = 0; j < k; ++j)
      if (kcol[j] < 0 || kcol[j] >= c1) return fail(CMPS_ERR_STATE, "unit cell: bond map");
    int32_t *d_rsig, *d_csig;
    int64_t *d_rdst, *d_cdst, *d_kcol;
    double *d_kscale, *d_cscale;
    CMPS_TRY(alloc(&d_rsig, sizeof(int32_t) * R));
    CMPS_TRY(alloc(&d_csig, sizeof(int32_t) * C));
    CMPS_TRY(alloc(&d_rdst, sizeof(int64_t) * R));
    CMPS_TRY(alloc(&d_cdst, sizeof(int64_t) * C));
    CMPS_TRY(alloc(&d_kcol, sizeof(int64_t) * k));
    CMPS_TRY(alloc(&d_kscale, sizeof(double) * k));
    CMPS_TRY(alloc(&d_cscale, sizeof(double) * C));
    CMPS_TRY(copy_wait(d_rsig, rsig.data(), sizeof(int32_t) * R, cudaMemcpyHostToDevice, st));
    CMPS_TRY(copy_wait(d_csig, csig.data(), sizeof(int32_t) * C, cudaMemcpyHostToDevice, st));
    CMPS_TRY(copy_wait(d_rdst, rdst.data(), sizeof(int64_t) * R, cudaMemcpyHostToDevice, st));
    CMPS_TRY(copy_wait(d_cdst, cdst_c.data(), sizeof(int64_t) * C, cudaMemcpyHostToDevice, st));
    CMPS_TRY(copy_wait(d_kcol, kcol.data(), sizeof(int64_t) * k, cudaMemcpyHostToDevice, st));
    CMPS_TRY(copy_wait(d_kscale, kscale.data(), sizeof(double) * k, cudaMemcpyHostToDevice, st));
    CMPS_TRY(copy_wait(d_cscale, cscale.data(), sizeof(double) * C, cudaMemcpyHostToDevice, st));
    // A0[s1][a0, a1] = U_m[(s1, a0), j]
    k_scatter_cell<<<grid_of(R * k), 256, 0, st>>>(S.U.re() + S.uoff[m], S.U.im() + S.uoff[m], R, k, d_rsig,
                                                   nullptr, d_rdst, d_kcol, nullptr, nullptr, c.A0, c0, c0 * c1);
    // A1[s2][a1, a2] = s[a1] V^dagger_m[j, (s2, a2)] / lambda_prev[a2]
    k_scatter_cell<<<grid_of(k * C), 256, 0, st>>>(S.Vd.re() + S.voff[m], S.Vd.im() + S.voff[m], k, C, nullptr,
                                                   d_csig, d_kcol, d_cdst, d_kscale, d_cscale, c.A1, c1, c1 * c0);
    CMPS_CUDA(cudaGetLastError());
  }

  // ---- dominant fixed points, on the charge blocks of the end bond ----
  const int64_t n = c0 * c0;
  cplx *w01, *w11, *w10, *lft, *rgt;
  CMPS_TRY(alloc(&w01, sizeof(cplx) * c0 * c1));
  CMPS_TRY(alloc(&w11, sizeof(cplx) * c1 * c1));
  CMPS_TRY(alloc(&w10, sizeof(cplx) * c1 * c0));
  CMPS_TRY(alloc(&lft, sizeof(cplx) * n));
  CMPS_TRY(alloc(&rgt, sizeof(cplx) * n));
  BlockMaps bm;
  struct BmFree {
    BlockMaps& m;
    ~BmFree() { m.release(); }
  } bm_free{bm};
  CMPS_TRY(build_block_maps(S, lam, inv_prev, st, bm));
  const int64_t nb = bm.nb;
  const int kd = std::max(2, std::min<int>(kdim, (int)std::min<int64_t>(nb, 64)));
  cplx *V, *hvec, *xl, *xr;
  int64_t* d_dense;
  CMPS_TRY(alloc(&V, sizeof(cplx) * (kd + 1) * nb));
  CMPS_TRY(alloc(&hvec, sizeof(cplx) * (kd + 1)));
  CMPS_TRY(alloc(&xl, sizeof(cplx) * nb));
  CMPS_TRY(alloc(&xr, sizeof(cplx) * nb));
  CMPS_TRY(alloc(&d_dense, sizeof(int64_t) * nb));
  CMPS_TRY(copy_wait(d_dense, bm.dense_of.data(), sizeof(int64_t) * nb, cudaMemcpyHostToDevice, st));
  {
    // start: the identity (the fixed point of a canonical cell), block by block
    std::vector<cplx> id((size_t)nb, kZero);
    for (size_t s = 0; s < bm.boff.size(); ++s)
      for (int64_t i = 0; i < bm.bdim[s]; ++i) id[bm.boff[s] + i * bm.bdim[s] + i] = kOne;
    CMPS_TRY(copy_wait(xl, id.data(), sizeof(cplx) * nb, cudaMemcpyHostToDevice, st));
    CMPS_TRY(copy_wait(xr, id.data(), sizeof(cplx) * nb, cudaMemcpyHostToDevice, st));
  }
  zc eta_l = 0.0, eta_r = 0.0;
  CMPS_TRY(dominant(bl, st, nb, [&](const cplx* in, cplx* out) { return apply_block_map(bm, true, in, out, st); },
                    tol, kd, 200, xl, V, hvec, &eta_l));
  CMPS_TRY(dominant(bl, st, nb, [&](const cplx* in, cplx* out) { return apply_block_map(bm, false, in, out, st); },
                    tol, kd, 200, xr, V, hvec, &eta_r));
  // the block-diagonal fixed points as dense chi0 x chi0 (column-major [bra, ket] / [ket, bra])
  CMPS_CUDA(cudaMemsetAsync(lft, 0, sizeof(cplx) * n, st));
  CMPS_CUDA(cudaMemsetAsync(rgt, 0, sizeof(cplx) * n, st));
  k_scatter_index<<<grid_of(nb), 256, 0, st>>>(xl, d_dense, nb, lft);
  k_scatter_index<<<grid_of(nb), 256, 0, st>>>(xr, d_dense, nb, rgt);
  CMPS_CUDA(cudaGetLastError());
  for (zc e : {eta_l, eta_r})
    if (std::abs(e.imag()) >= 1e-10 * std::abs(e.real()) || !(e.real() > 0.0))
      return fail(CMPS_ERR_SOLVER, "unit cell: dominant transfer-matrix eigenvalue is not real and positive");
  for (cplx* v : {lft, rgt}) {
    const zc tr = trace_of(v, c0, st);
    if (!(std::abs(tr) > 0.0)) return fail(CMPS_ERR_SOLVER, "unit cell: traceless fixed point");
    const zc ph = std::conj(tr) / std::abs(tr);
    k_hermitize<<<grid_of(n), 256, 0, st>>>(v, c0, make_cuDoubleComplex(ph.real(), ph.imag()));
  }

  // ---- SqrtDR of the left fixed point; Lambda'^2 = eig(X r X^dag) ----
  {
    cplx* E;
    double* w;
    int* dinfo;
    CMPS_TRY(alloc(&E, sizeof(cplx) * n));
    CMPS_TRY(alloc(&w, sizeof(double) * c0));
    CMPS_TRY(alloc(&dinfo, sizeof(int)));
    CMPS_CUDA(cudaMemcpyAsync(E, lft, sizeof(cplx) * n, cudaMemcpyDeviceToDevice, st));
    cusolverDnSetStream(sol, st);
    int lwork = 0;
    if (cusolverDnZheevd_bufferSize(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, (int)c0, E, (int)c0, w,
                                    &lwork) != CUSOLVER_STATUS_SUCCESS)
      return fail(CMPS_ERR_SOLVER, "unit cell: zheevd buffer query failed");
    cplx* work;
    CMPS_TRY(alloc(&work, sizeof(cplx) * std::max(1, lwork)));
    if (cusolverDnZheevd(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, (int)c0, E, (int)c0, w, work, lwork,
                         dinfo) != CUSOLVER_STATUS_SUCCESS)
      return fail(CMPS_ERR_SOLVER, "unit cell: zheevd failed");
    std::vector<double> hw(c0);
    int info = 0;
    cudaMemcpyAsync(hw.data(), w, sizeof(double) * c0, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&info, dinfo, sizeof(int), cudaMemcpyDeviceToHost, st);
    CMPS_CUDA(cudaStreamSynchronize(st));
    if (info != 0) return fail(CMPS_ERR_SOLVER, "unit cell: zheevd did not converge");
    double mx = 0.0;
    for (double x : hw) mx = std::max(mx, std::fabs(x));
    const double cut = mx * 100.0 * kEps;
    std::vector<int32_t> keep;
    std::vector<double> root;
    int neg = 0;
    for (int64_t i = 0; i < c0; ++i)
      if (std::fabs(hw[i]) > cut) {
        keep.push_back((int32_t)i);
        root.push_back(std::sqrt(std::fabs(hw[i])));
        if (hw[i] < 0.0) ++neg;
      }
    if (keep.empty() || (neg != 0 && neg != (int)keep.size()))
      return fail(CMPS_ERR_SOLVER, "unit cell: SqrtDR failure (eigenvalues of both signs)");
    const int64_t kl = (int64_t)keep.size();
    int32_t* d_keep;
    double* d_root;
    cplx *X, *XR, *B;
    CMPS_TRY(alloc(&d_keep, sizeof(int32_t) * kl));
    CMPS_TRY(alloc(&d_root, sizeof(double) * kl));
    CMPS_TRY(alloc(&X, sizeof(cplx) * kl * c0));
    CMPS_TRY(alloc(&XR, sizeof(cplx) * kl * c0));
    CMPS_TRY(alloc(&B, sizeof(cplx) * kl * kl));
    CMPS_TRY(copy_wait(d_keep, keep.data(), sizeof(int32_t) * kl, cudaMemcpyHostToDevice, st));
    CMPS_TRY(copy_wait(d_root, root.data(), sizeof(double) * kl, cudaMemcpyHostToDevice, st));
    k_make_x<<<grid_of(kl * c0), 256, 0, st>>>(E, c0, d_keep, d_root, kl, X);
    bl.gemm(CUBLAS_OP_N, CUBLAS_OP_N, kl, c0, c0, kOne, X, kl, rgt, c0, kZero, XR, kl);
    bl.gemm(CUBLAS_OP_N, CUBLAS_OP_C, kl, kl, c0, kOne, XR, kl, X, kl, kZero, B, kl);
    if (bl.st != CMPS_OK) return bl.st;
    double* wb;
    CMPS_TRY(alloc(&wb, sizeof(double) * kl));
    int lw2 = 0;
    if (cusolverDnZheevd_bufferSize(sol, CUSOLVER_EIG_MODE_NOVECTOR, CUBLAS_FILL_MODE_LOWER, (int)kl, B, (int)kl, wb,
                                    &lw2) != CUSOLVER_STATUS_SUCCESS)
      return fail(CMPS_ERR_SOLVER, "unit cell: zheevd buffer query failed");
    cplx* work2;
    CMPS_TRY(alloc(&work2, sizeof(cplx) * std::max(1, lw2)));
    if (cusolverDnZheevd(sol, CUSOLVER_EIG_MODE_NOVECTOR, CUBLAS_FILL_MODE_LOWER, (int)kl, B, (int)kl, wb, work2, lw2,
                         dinfo) != CUSOLVER_STATUS_SUCCESS)
      return fail(CMPS_ERR_SOLVER, "unit cell: zheevd failed");
    std::vector<double> hb(kl);
    cudaMemcpyAsync(hb.data(), wb, sizeof(double) * kl, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&info, dinfo, sizeof(int), cudaMemcpyDeviceToHost, st);
    CMPS_CUDA(cudaStreamSynchronize(st));
    if (info != 0) return fail(CMPS_ERR_SOLVER, "unit cell: zheevd did not converge");
    double sum = 0.0, bmax = 0.0;
    for (double x : hb) {
      if (x > 0.0) sum += x;
      bmax = std::max(bmax, x);
    }
    if (!(sum > 0.0)) return fail(CMPS_ERR_SOLVER, "unit cell: no weight in the new boundary values");
    double ent = 0.0;
    int64_t chi_new = 0;
    for (double x : hb) {
      if (!(x > 0.0)) continue;
      const double p = x / sum;
      ent -= p * std::log(p);
      if (x > 1e-14 * bmax) ++chi_new;
    }
    out->entropy = ent;
    out->chi = chi_new;
  }

  // ---- energy per vertex from trace tables ----
  // F[s1',s1] = A0[s1']^H l A0[s1] (c1 x c1), G[s2,s2'] = A1[s2] r A1[s2']^H,
  // T1[(s1',s1),(s2,s2')] = Tr[F G]; P[s2',s2] = A1[s2']^H K A1[s2] with
  // K = sum F[s1,s1], Q[s1,s1'] = A0[s1] Gs A0[s1']^H with Gs = sum G[s2,s2],
  // T2[(s2',s2),(s1,s1')] = Tr[P Q].  Pair index (a, b) -> a + d b.
  const int64_t dd = (int64_t)d * d;
  cplx *F, *G, *FT, *P, *Q, *PT, *T1, *T2, *K, *Gs;
  CMPS_TRY(alloc(&F, sizeof(cplx) * dd * c1 * c1));
  CMPS_TRY(alloc(&G, sizeof(cplx) * dd * c1 * c1));
  CMPS_TRY(alloc(&FT, sizeof(cplx) * dd * c1 * c1));
  CMPS_TRY(alloc(&P, sizeof(cplx) * dd * c0 * c0));
  CMPS_TRY(alloc(&Q, sizeof(cplx) * dd * c0 * c0));
  CMPS_TRY(alloc(&PT, sizeof(cplx) * dd * c0 * c0));
  CMPS_TRY(alloc(&T1, sizeof(cplx) * dd * dd));
  CMPS_TRY(alloc(&T2, sizeof(cplx) * dd * dd));
  CMPS_TRY(alloc(&K, sizeof(cplx) * c1 * c1));
  CMPS_TRY(alloc(&Gs, sizeof(cplx) * c1 * c1));
  for (int s1 = 0; s1 < d; ++s1) {
    bl.gemm(CUBLAS_OP_N, CUBLAS_OP_N, c0, c1, c0, kOne, lft, c0, c.a0(s1), c0, kZero, w01, c0);  // l A0[s1]
    for (int s1p = 0; s1p < d; ++s1p)
      bl.gemm(CUBLAS_OP_C, CUBLAS_OP_N, c1, c1, c0, kOne, c.a0(s1p), c0, w01, c0, kZero,
              F + (s1p + (int64_t)d * s1) * c1 * c1, c1);
  }
  for (int s2 = 0; s2 < d; ++s2) {
    bl.gemm(CUBLAS_OP_N, CUBLAS_OP_N, c1, c0, c0, kOne, c.a1(s2), c1, rgt, c0, kZero, w10, c1);  // A1[s2] r
    for (int s2p = 0; s2p < d; ++s2p)
      bl.gemm(CUBLAS_OP_N, CUBLAS_OP_C, c1, c1, c0, kOne, w10, c1, c.a1(s2p), c1, kZero,
              G + (s2 + (int64_t)d * s2p) * c1 * c1, c1);
  }
  if (bl.st != CMPS_OK) return bl.st;
  CMPS_CUDA(cudaMemsetAsync(K, 0, sizeof(cplx) * c1 * c1, st));
  CMPS_CUDA(cudaMemsetAsync(Gs, 0, sizeof(cplx) * c1 * c1, st));
  for (int s = 0; s < d; ++s) {
    if (cublasZaxpy(bl.h, (int)(c1 * c1), &kOne, F + (s + (int64_t)d * s) * c1 * c1, 1, K, 1) !=
            CUBLAS_STATUS_SUCCESS ||
        cublasZaxpy(bl.h, (int)(c1 * c1), &kOne, G + (s + (int64_t)d * s) * c1 * c1, 1, Gs, 1) !=
            CUBLAS_STATUS_SUCCESS)
      return fail(CMPS_ERR_CUDA, "unit cell: axpy failed");
  }
  for (int s2 = 0; s2 < d; ++s2) {
    bl.gemm(CUBLAS_OP_N, CUBLAS_OP_N, c1, c0, c1, kOne, K, c1, c.a1(s2), c1, kZero, w10, c1);  // K A1[s2]
    for (int s2p = 0; s2p < d; ++s2p)
      bl.gemm(CUBLAS_OP_C, CUBLAS_OP_N, c0, c0, c1, kOne, c.a1(s2p), c1, w10, c1, kZero,
              P + (s2p + (int64_t)d * s2) * c0 * c0, c0);
  }
  for (int s1 = 0; s1 < d; ++s1) {
    bl.gemm(CUBLAS_OP_N, CUBLAS_OP_N, c0, c1, c1, kOne, c.a0(s1), c0, Gs, c1, kZero, w01, c0);  // A0[s1] Gs
    for (int s1p = 0; s1p < d; ++s1p)
      bl.gemm(CUBLAS_OP_N, CUBLAS_OP_C, c0, c0, c1, kOne, w01, c0, c.a0(s1p), c0, kZero,
              Q + (s1 + (int64_t)d * s1p) * c0 * c0, c0);
  }
  if (bl.st != CMPS_OK) return bl.st;
  // Tr[F G] = vec(F^T) . vec(G): T1 = FT_mat^T G_mat over the stacked matrices
  k_transpose_stack<<<grid_of(dd * c1 * c1), 256, 0, st>>>(F, FT, c1, dd);
  k_transpose_stack<<<grid_of(dd * c0 * c0), 256, 0, st>>>(P, PT, c0, dd);
  bl.gemm(CUBLAS_OP_T, CUBLAS_OP_N, dd, dd, c1 * c1, kOne, FT, c1 * c1, G, c1 * c1, kZero, T1, dd);
  bl.gemm(CUBLAS_OP_T, CUBLAS_OP_N, dd, dd, c0 * c0, kOne, PT, c0 * c0, Q, c0 * c0, kZero, T2, dd);
  if (bl.st != CMPS_OK) return bl.st;
  // Contract the tables with the MPO blocks on the device.  Operator O[s', s]
  // as a pair vector: site 0 of a cell reads pairs (s', s) = s' + d s of the
  // first table index; site 1 reads pairs (s, s') = s + d s' of the second.
  // Columns of Cm: ColX_k in second-index order; of Rm: RowX_k in first-index
  // order.  V1 = T1 [Cm | e | h'] and V2 = T2 Cm, with e the identity pairs
  // (s, s) and h' = H1 in second-index order; everything else is dot products
  // of these few columns on the host.
  std::map<std::pair<int, int>, std::vector<zc>> blocks;
  for (const WEntry& e : W) {
    if (!((e.bl == D - 1 && e.br >= 0 && e.br <= D - 2) || (e.br == 0 && e.bl >= 1 && e.bl <= D - 1))) continue;
    auto& O = blocks[{e.bl, e.br}];
    if (O.empty()) O.assign((size_t)dd, 0.0);
    O[e.sp + (size_t)d * e.s] += zc(e.wr, e.wi);  // O[s', s]
  }
  auto second = [&](const std::vector<zc>& O) {  // O[s', s] at s + d s'
    std::vector<zc> v((size_t)dd);
    for (int sp = 0; sp < d; ++sp)
      for (int sv = 0; sv < d; ++sv) v[sv + (size_t)d * sp] = O[sp + (size_t)d * sv];
    return v;
  };
  std::vector<std::vector<zc>> Rcols, Ccols;
  for (int kb = 1; kb <= D - 2; ++kb) {
    auto r = blocks.find({D - 1, kb}), c2 = blocks.find({kb, 0});
    if (r == blocks.end() || c2 == blocks.end()) continue;
    Rcols.push_back(r->second);
    Ccols.push_back(second(c2->second));
  }
  std::vector<zc> H1((size_t)dd, 0.0);
  if (blocks.count({D - 1, 0})) H1 = blocks[{D - 1, 0}];
  std::vector<zc> ess((size_t)dd, 0.0);
  for (int sv = 0; sv < d; ++sv) ess[sv + (size_t)d * sv] = 1.0;
  const int64_t nk = (int64_t)Rcols.size();
  const int64_t ncol = nk + 2;
  std::vector<cplx> rhs((size_t)dd * ncol);
  auto put = [&](int64_t col, const std::vector<zc>& v) {
    for (int64_t p = 0; p < dd; ++p) rhs[p + (size_t)dd * col] = make_cuDoubleComplex(v[p].real(), v[p].imag());
  };
  for (int64_t k = 0; k < nk; ++k) put(k, Ccols[k]);
  put(nk, ess);
  put(nk + 1, second(H1));
  cplx *d_rhs, *V1, *V2;
  CMPS_TRY(alloc(&d_rhs, sizeof(cplx) * dd * ncol));
  CMPS_TRY(alloc(&V1, sizeof(cplx) * dd * ncol));
  CMPS_TRY(alloc(&V2, sizeof(cplx) * dd * std::max<int64_t>(1, nk)));
  CMPS_TRY(copy_wait(d_rhs, rhs.data(), sizeof(cplx) * dd * ncol, cudaMemcpyHostToDevice, st));
  bl.gemm(CUBLAS_OP_N, CUBLAS_OP_N, dd, ncol, dd, kOne, T1, dd, d_rhs, dd, kZero, V1, dd);
  if (nk) bl.gemm(CUBLAS_OP_N, CUBLAS_OP_N, dd, nk, dd, kOne, T2, dd, d_rhs, dd, kZero, V2, dd);
  if (bl.st != CMPS_OK) return bl.st;
  std::vector<cplx> hv1((size_t)dd * ncol), hv2((size_t)dd * std::max<int64_t>(1, nk));
  cudaMemcpyAsync(hv1.data(), V1, sizeof(cplx) * dd * ncol, cudaMemcpyDeviceToHost, st);
  if (nk) cudaMemcpyAsync(hv2.data(), V2, sizeof(cplx) * dd * nk, cudaMemcpyDeviceToHost, st);
  CMPS_CUDA(cudaStreamSynchronize(st));
  auto dot = [&](const std::vector<zc>& u, const std::vector<cplx>& M, int64_t col) {
    zc acc = 0.0;
    for (int64_t p = 0; p < dd; ++p) acc += u[p] * zc(M[p + (size_t)dd * col].x, M[p + (size_t)dd * col].y);
    return acc;
  };
  zc norm = dot(ess, hv1, nk);                       // sum_{s1,s2} T1[(s1,s1),(s2,s2)] = eta Tr[l r]
  zc local = dot(H1, hv1, nk) + dot(ess, hv1, nk + 1);  // H1 on site 0, on site 1
  zc bond1 = 0.0, bond2 = 0.0;
  for (int64_t k = 0; k < nk; ++k) {
    bond1 += dot(Rcols[k], hv1, k);   // RowX on site 0, ColX on site 1
    bond2 += dot(Rcols[k], hv2, k);   // RowX on site 1, ColX on the next cell's site 0
  }
  const double eta = eta_l.real();
  const zc e = 0.5 * (local + bond1 + bond2 / eta) / norm;
  out->energy = e.real();
  out->energy_imag = e.imag();
  out->eta_left = eta_l.real();
  out->eta_right = eta_r.real();
  return CMPS_OK;
}

}  // namespace cmps
