// Device-resident two-vertex effective Hamiltonian (internal).
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <vector>

#include "internal.h"
#include "kernels.h"

struct cmps_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  void* solver = nullptr;  // cusolverDnHandle_t, created on first SVD
  void* blas = nullptr;    // cublasHandle_t, created on first SVD (Gram matrices of big sectors)
  void* svd_pool = nullptr;  // worker streams and handles of the block SVD, created on first use
};

namespace cmps {

// Two-vertex wavefunction space: Theta = sum over middle charges m of dense
// blocks Theta_m[(sigma1, a0), (sigma2, a2)], q(sigma1)+q(a0) = m =
// q(a2)-q(sigma2).  Rows are grouped by sigma1 (each sigma1 contributes the
// whole a0-sector of charge m - q(sigma1)), columns by sigma2 (a2-sector of
// charge m + q(sigma2)); the states appear class by class (Heff::cls_mem),
// and blocks are row-major.
struct ThetaSpace {
  std::vector<QKey> mq;                     // middle charges
  std::map<QKey, int> mfind;
  std::vector<int64_t> nrows, ncols, base;  // per m
  std::vector<std::vector<int64_t>> rowoff, coloff;  // [m][sigma] -> offset or -1
  int64_t total = 0;
  int find(const QKey& q) const {
    auto it = mfind.find(q);
    return it == mfind.end() ? -1 : it->second;
  }
};

struct SvdResult;
struct SplitState;
struct Canon;
struct CanonTc;

struct Heff {
  cmps_context* ctx = nullptr;
  int device = 0;                // copied from ctx at build: valid even if ctx is destroyed first
  Rules rules;
  int d = 0;
  std::vector<QKey> sigq;       // basis charges
  // Charge classes of the physical index: the states of one charge, classes
  // in first-seen order, states in basis order.  Theta rows and columns are
  // grouped by class, so a class's states are equally strided in a block.
  std::vector<std::vector<int>> cls_mem;
  std::vector<int> cls_of, cls_pos;  // state -> class, position inside it
  Env L, R;                     // environments (device)
  std::vector<WEntry> W;        // non-zero MPO entries
  int D = 0;
  std::vector<QKey> bq;         // MPO bond charges
  std::vector<int16_t> bq_raw;  // as given (for export)
  ThetaSpace th;
  int64_t n_allowed = 0, full_length = 0;
  // ARPACK-order maps, generated on the device from per-column and per-sector
  // descriptors (a few thousand entries instead of n host-side ones)
  struct MapCol {
    int64_t colpart, colth, start;  // s2 + d a2; theta column in its block; first ARPACK index
    int64_t m;
  };
  struct MapSec {
    int64_t rowstart, nrows, base, ncols;  // rows of block m in ARPACK row order
  };
  std::vector<MapCol> map_cols;
  std::vector<MapSec> map_secs;
  std::vector<int64_t> map_rowlin, map_rowth;  // per allowed row: s1 + d a0, theta row
  // mode 0: ARPACK index -> theta offset; mode 1: -> full linear index
  int arpack_map(int mode, int64_t* d_out, cudaStream_t st) const;
  int allowed_indices(int64_t* host_out) const;
  // ARPACK order <-> sector blocks as 32 x 32 transpose tiles: a group is up
  // to 32 ARPACK columns of one (block m, sigma2) with consecutive a2
  // positions, i.e. consecutive theta columns.
  struct PackGroup {
    int64_t off;  // into the group column list
    int32_t cnt, m;
  };
  struct PackTile {
    int32_t group, r0;
  };
  void* d_pack = nullptr;        // one allocation: cols, secs, rowth, group columns, groups, tiles
  const MapCol* d_map_cols = nullptr;
  const MapSec* d_map_secs = nullptr;
  const int64_t* d_map_rowth = nullptr;
  const int32_t* d_pack_gcols = nullptr;
  const PackGroup* d_pack_groups = nullptr;
  const PackTile* d_pack_tiles = nullptr;
  int64_t n_pack_tiles = 0;
  int build_pack(cudaStream_t st);
  // in: n_allowed interleaved complex (ARPACK order) -> theta blocks, and back
  int pack(const double* in, const Planar& out, cudaStream_t st) const;
  int unpack(const Planar& in, double* out, cudaStream_t st) const;
  // LeftPart / RightPart sector blocks
  Planar LP, RP;
  std::vector<AxpyBlock> lp_blocks, rp_blocks;
  std::vector<AxpyTerm> lp_terms, rp_terms;
  AxpyBlock* d_lp_blocks = nullptr;
  AxpyTerm* d_lp_terms = nullptr;
  AxpyBlock* d_rp_blocks = nullptr;
  AxpyTerm* d_rp_terms = nullptr;
  std::map<std::array<int, 4>, int64_t> lp_off, rp_off;  // (b1, sigma', sigma, sector) -> offset
  std::vector<int64_t> t_base;   // [b1 * nm + m] -> offset into T, -1 if absent
  Planar T;                      // stage-1 intermediate, allocated on first use (ensure_T)
  int64_t t_len = 0;             // its length in complex elements
  int ensure_T();
  GemmPlan stage1, stage2;
  // Output sectors this matvec computes (1 = owned).  All of them, unless the
  // matvec is sharded across GPUs by output sector; then the output blocks
  // of the other sectors are left unwritten and only the theta-layout entry
  // points apply.  sector_flops: executed flops per output sector.
  std::vector<uint8_t> owned;
  std::vector<double> sector_flops;
  int build_plans();
  int set_owned(const uint8_t* mask);
  bool all_owned() const;
  // Windows of the theta-layout entry point, for a sharded matvec whose ranks
  // hold only part of the vectors: input sector m is read at in_base[m] of an
  // input of in_len entries per plane, owned output sector m' is written at
  // out_base[m'] of an output of out_len.  By default both are the theta
  // layout itself.  in_need: the input sectors the owned outputs read.
  std::vector<int64_t> in_base, out_base;
  int64_t in_len = 0, out_len = 0;
  bool windowed = false;
  std::vector<uint8_t> in_need;
  int set_windows(const int64_t* in_base, int64_t in_len, const int64_t* out_base, int64_t out_len);
  void default_windows();
  // every sector owned and the vectors in the theta layout: the whole-vector
  // entry points (ARPACK order, eigensolver, adjoint) apply
  bool whole() const { return all_owned() && !windowed; }
  // Excited-state projectors (TwoVertexComponents::ProjectorTensors,
  // DMRG_routines.hpp:205): the matvec adds sum_p w_p (P_p . x) conj(P_p),
  // the bilinear product P . x taken without conjugation
  // (DMRG_routines.cpp:947-973).  Stored as phi_p = conj(P_p) in the theta
  // layout (vector p: re plane at proj.d + 2 p n, im plane n further), so the
  // term is sum_p w_p phi_p <phi_p, x>.
  Planar proj;
  int proj_np = 0;
  double* d_proj = nullptr;  // weights [np], coefficients [2 np + 4]
  std::vector<double> proj_w;
  // Measured tile shapes of the grouped GEMM plans the handle's matvec runs
  // (autotune_plan); the tcgen05 split stages have fixed tiles.
  int autotune(TuneStats* stats);
  int set_projectors(int np, const double* host_arpack, const double* weights);
  // the same from device vectors phi_p = conj(P_p), ARPACK order, interleaved
  int set_projectors_device(int np, const double* d_phi_arpack, const double* weights);
  int add_projectors(const Planar& in, Planar& out, cudaStream_t st);
  double flops_canonical = 0.0, flops_executed = 0.0;
  // Contraction order of the FP64 matvec: folded (LeftPart / RightPart, the
  // two stages above) or canonical (L, W1, W2, R one index at a time,
  // canonical.cu).  order_req is what the caller asked for (CMPS_ORDER_*),
  // order the one in use; flops_folded / flops_canon are the executed flops
  // of each order.
  int order_req = CMPS_ORDER_AUTO, order = CMPS_ORDER_FOLDED;
  double flops_folded = 0.0, flops_canon = 0.0;
  Canon* canon = nullptr;
  int select_order();
  // The split-precision operator runs the canonical order instead of the
  // folded order on tcgen05 (split_tf32.cu): on tcgen05 in split BF16 when
  // ctc is set (canonical_tc.cu), else in FP32 (canonical.cu).
  bool low_canonical = false;
  CanonTc* ctc = nullptr;
  int precision = CMPS_FP64;
  SplitState* split = nullptr;   // split-TF32 operands and plans (split_tf32.cu)
  // work vectors
  Planar x, y;                   // theta-space vectors
  double* d_io = nullptr;        // interleaved staging (2 * n_allowed doubles)
  bool have_theta = false;
  Planar theta;                  // last eigenvector (theta space)
  // Krylov basis: vector j at kv.d + 2 j n (n = th.total), its real plane
  // then its imaginary plane, so each basis vector is itself a Planar view
  Planar kv;
  int kv_dim = 0;
  VecOps ops;
  double* h_ab = nullptr;        // pinned: alpha_j, beta_j of the current Lanczos step
  // Work of the last eigs() call.
  struct EigStats {
    int mv_split = 0, mv_fp64 = 0, cycles = 0;
    double ms_split = 0.0, ms_fp64 = 0.0, ms_total = 0.0;
  } eig_stats;

  ~Heff();
  int build(cmps_context* c, const Rules& r, const cmps_mpx_desc* Ld, const cmps_mpx_desc* Wd,
            const cmps_mpx_desc* Rd);
  int build_from_envs(cmps_context* c, const Rules& r, const Env& Lsrc, const cmps_mpx_desc* Wd, const Env& Rsrc);
  int parse_mpo(const cmps_mpx_desc* Wd);
  int finish();  // sector structure, LeftPart/RightPart, GEMM plans (L, R, W set)
  int apply_theta(const Planar& in, Planar& out, cudaStream_t st);  // theta-space matvec
  int apply_theta_fp64(const Planar& in, Planar& out, cudaStream_t st);   // with the projectors
  int apply_fp64_stages(const Planar& in, Planar& out, cudaStream_t st);  // the GEMM stages only (order in use)
  int apply_folded_fp64(const Planar& in, Planar& out, cudaStream_t st);  // the two folded stages
  int apply_stage(int which, const Planar& in, Planar& out, cudaStream_t st);  // 1: T = LP in, 2: out = T RP
  int apply_host(const double* in, double* out);
  int apply_device(const double* din, double* dout, cudaStream_t st);
  // start_in_x: the start vector is already in x (theta layout, device)
  int eigs(const double* guess, double tol, int max_restarts, int kdim, double* eval, double* evec,
           int* matvecs, bool start_in_x = false);
};

// Result of the charge-block SVD of theta (svd.cu).
struct SvdResult {
  uint64_t serial = 0;  // unique per factorisation of a DMRG run (cache keys)
  Rules rules;
  int d = 0;
  std::vector<QKey> sigq;
  Bond a0, a2;
  ThetaSpace th;
  std::vector<int64_t> kept;            // per m
  std::vector<int64_t> uoff, voff;      // per m, offsets into U / Vd
  Planar U, Vd;                         // U_m: nrows[m] x kept[m]; Vd_m: kept[m] x ncols[m] (row-major)
  std::vector<double> values;           // kept, global descending order
  std::vector<std::pair<int, int64_t>> order;  // global index -> (m, j)
  std::vector<std::vector<int64_t>> gidx;      // [m][j] -> global index
  double discarded = 0.0;
  int routes[3] = {0, 0, 0};  // sectors factored exactly, by the Gram matrix, by the randomized route
};

// kept_hint (optional): per middle charge, the values a previous
// factorisation kept; it sizes the randomized route's range.
int theta_svd(Heff& H, int64_t chi, double max_trunc, SvdResult& out,
              const std::map<QKey, int64_t>* kept_hint = nullptr);
// adjoint.cu: derivative of the contraction with respect to a vertex coupling
int parse_derivative_mpo(const Heff& H, const cmps_mpx_desc* dW, std::vector<WEntry>& out);
// W gains a zero-weight entry at every position where dW is non-zero and W
// is not, so that LeftPart / RightPart blocks exist for every dW term.
void extend_pattern(std::vector<WEntry>& W, const std::vector<WEntry>& dW);
int derivative_parts(Heff& H, const std::vector<WEntry>& dW, const Env* dL, const Env* dR, Planar& LPd,
                     Planar& RPd);
int heff_adjoint(Heff& H, const std::vector<WEntry>& dW, const Env* dL, const Env* dR, double* grad);
int growth_fidelity(Heff& H, const SvdResult& s, const std::vector<double>& lam, const std::vector<double>& prev,
                    double* out);
int sweep_fidelity(Heff& H, const SvdResult& s, const std::vector<double>& lam, const Planar& guess, double* out);
int left_update(Heff& H, const SvdResult& s, Env& out);
int right_update(Heff& H, const SvdResult& s, Env& out);
int derivative_envs(Heff& H, const SvdResult& s, const std::vector<WEntry>& dW, const Env* dL, const Env* dR,
                    Env& dLn, Env& dRn);

// The canonical contraction order (canonical.cu).
// the FP64 form's intermediates (X/Z and Y), which the split forms borrow
int canonical_scratch(const Heff& H, const Planar** xz, const Planar** y);
// need (optional): the theta sectors the canonical order's first stage reads
int canonical_flops(const Heff& H, double* flops, std::vector<uint8_t>* need = nullptr);
// measured tile shapes of the canonical plans (FP32 or FP64 launches)
int autotune_canonical(Heff& H, bool fp32, cudaStream_t st, TuneStats* stats);
int build_canonical(Heff& H);
void release_canonical(Heff* h);
// which: 1 = stages L and W1, 2 = stages W2 and R, 0 = all four
int apply_canonical(Heff& H, int which, const Planar& in, Planar& out, cudaStream_t st);
// the same in FP32 (FP32 copies of the operands built by build_canonical32)
int build_canonical32(Heff& H);
int apply_canonical32(Heff& H, int which, const Planar& in, Planar& out, cudaStream_t st);

// The canonical order in split BF16 on tcgen05 (canonical_tc.cu): whole
// vectors only (no windows, every sector owned).
int build_canonical_tc(Heff& H);
void release_canonical_tc(Heff* h);
// which: 1 = theta in, stages R and W2; 2 = stages W1 and L; 0 = all four
int apply_canonical_tc(Heff& H, int which, const Planar& in, Planar& out, cudaStream_t st);
void canonical_tc_error_words(const Heff& H, int** d_err, int** h_err);
// executed complex flops of one matvec, padding included
double canonical_tc_flops(const Heff& H);

// Split-precision operands for the tcgen05 path (split_tf32.cu).
int prepare_precision(Heff* h, int precision);
void release_split(Heff* h);
int apply_split(Heff& H, const Planar& in, Planar& out, cudaStream_t st);
// The same matvec without a host synchronisation; a pipeline time-out is
// recorded in the handle's error word, cleared by split_reset_error() and
// read by split_error().
int apply_split_async(Heff& H, const Planar& in, Planar& out, cudaStream_t st);
int split_reset_error(Heff& H, cudaStream_t st);
int apply_split_stage(Heff& H, int which, const Planar& in, Planar& out, cudaStream_t st);
int split_error(Heff& H);
// The form of the handle's split operator (CMPS_FORM_*).
int split_form(const Heff& H);
// cuSOLVER handle owned by the context (svd.cu).
void release_solver(cmps_context* ctx);
// The context's cuBLAS / cuSOLVER handles, bound to its stream (svd.cu).
int context_blas(cmps_context* ctx, void** out);
int context_solver(cmps_context* ctx, void** out);

// iDMRG unit cell of a growth step (unitcell.cu): Orthogonalise +
// iTwoVertexEnergy from the step's factors U, s, V^dagger (S, lam: the
// rescaled values) and the previous step's values lam_prev.
struct UnitCellMeasure {
  double energy = 0.0, energy_imag = 0.0;  // per vertex
  double entropy = 0.0;                     // of the new boundary values Lambda'
  double eta_left = 0.0, eta_right = 0.0;   // dominant transfer-matrix eigenvalues
  int64_t chi = 0;                          // Lambda' values above 1e-14 of the largest (squared)
};
int unit_cell_measure(cmps_context* ctx, const SvdResult& S, const std::vector<double>& lam,
                      const std::vector<double>& lam_prev, const std::vector<WEntry>& W, int D, double tol, int kdim,
                      UnitCellMeasure* out);

int copy_env(const Env& src, Env& dst, cudaStream_t st);

int build_env_from_desc(const Rules& r, const cmps_mpx_desc* desc, bool right, Env& env, int D,
                        const std::vector<QKey>& bq, cudaStream_t st);
int parse_index_charges(const Rules& r, const cmps_mpx_desc* desc, int idx, std::vector<QKey>& out);

// Excited-state projectors from stored states (projector.cu; ProjectorBlocks,
// DMRG_routines.cpp:446-581).  A stored state is a snapshot of a finite
// chain's state: its left tensors lsvd[1..nleft], the window's factors with
// its values and its right tensors rsvd[1..length - nleft - 2].
struct ProjectedState;
int projected_state_create(cmps_context* ctx, const std::map<int64_t, std::shared_ptr<SvdResult>>& lsvd,
                           const std::map<int64_t, std::shared_ptr<SvdResult>>& rsvd, const SvdResult& window,
                           const std::vector<double>& lambda, int64_t nleft, int64_t length, double weight,
                           ProjectedState** out);
void projected_state_destroy(ProjectedState* p);
// The projector tensor of every stored state for H's window (the current
// state's tensors lsvd / rsvd), installed as H's projectors.
int install_projectors(cmps_context* ctx, std::vector<ProjectedState*>& states,
                       const std::map<int64_t, std::shared_ptr<SvdResult>>& lsvd,
                       const std::map<int64_t, std::shared_ptr<SvdResult>>& rsvd, int64_t nleft, int64_t length,
                       Heff& H);

}  // namespace cmps

struct cmps_heff {
  std::unique_ptr<cmps::Heff> impl;
};

struct cmps_block {
  cmps::Rules rules;
  cmps::Env env;
  ~cmps_block() { env.data.release(); }
};
