/*
 * chainamps_b200 -- C ABI of the B200 implementation of the ChainAMPS
 * two-site DMRG hot path (effective-Hamiltonian matvec, Krylov ground state,
 * charge-block SVD truncation, environment updates).
 *
 * Every entry point returns an int status (CMPS_OK == 0) and never aborts;
 * cmps_last_error() gives a one-line description of the last failure on the
 * calling thread.  Complex numbers are interleaved (re, im) doubles, exactly
 * std::complex<double> as the reference stores them.  Tensors cross the
 * boundary in the reference's own storage: an MPX_matrix is a list of
 * directed, charge-labelled indices plus one CSC matrix whose rows combine the
 * first num_row_indices indices and whose columns combine the rest, first
 * index fastest (MPX_matrix.cpp:219-236, MPXIndex.cpp:8-24,
 * sparse_interface.cpp:85-91).  Charges are QuantumNumberInt (short)
 * (common_defs.hpp:20); Z_N charges add modulo N, N <= 0 means Z
 * (states.hpp:176-206).
 */
#ifndef CHAINAMPS_B200_H
#define CHAINAMPS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  CMPS_OK = 0,
  CMPS_ERR_ARG = 1,        /* bad argument / inconsistent shapes */
  CMPS_ERR_CHARGE = 2,     /* a stored entry violates charge conservation */
  CMPS_ERR_CUDA = 3,       /* CUDA runtime / driver failure */
  CMPS_ERR_NOMEM = 4,      /* device allocation failed */
  CMPS_ERR_SOLVER = 5,     /* eigensolver / SVD did not converge */
  CMPS_ERR_STATE = 6       /* call out of order (e.g. no eigenvector yet) */
};

enum {
  CMPS_FP64 = 0,           /* all contraction arithmetic in complex double */
  CMPS_SPLIT_TF32 = 1,     /* contractions as 3-term split TF32 on tcgen05, FP32 accumulate */
  CMPS_SPLIT_BF16 = 2      /* contractions as 3-term split BF16 (hi + mid) on tcgen05, FP32
                              accumulate: about twice the split-TF32 rate, operands held to
                              16 significant bits (matvec error ~1e-5 relative); the mixed
                              eigensolver refines with FP64 cycles as for split-TF32 */
};

/* Contraction order of the FP64 matvec.  Folded: the reference's
 * (LeftPart . V) . RightPart, W folded into the environments
 * (DMRG_routines.cpp:779, :943).  Canonical: L . theta, then W on sigma1,
 * W on sigma2, then . R, one index at a time -- the same operator, far fewer
 * flops for a vertex with many states per charge and dense operators.
 * Auto (the default) takes the canonical order when it executes at most half
 * the folded order's flops. */
enum {
  CMPS_ORDER_AUTO = 0,
  CMPS_ORDER_FOLDED = 1,
  CMPS_ORDER_CANONICAL = 2
};

/* Form of a handle's split-precision operator (cmps_heff_split_form).  The
 * canonical order is taken when it executes at most a quarter of the folded
 * order's flops; split BF16 runs it on tcgen05 (whole vectors only; a
 * sharded or windowed handle, split TF32, or a device without room for the
 * BF16 intermediates runs it in FP32). */
enum {
  CMPS_FORM_NONE = 0,            /* FP64 handle: no split operator */
  CMPS_FORM_FOLDED_TC = 1,       /* folded order, two tcgen05 stages */
  CMPS_FORM_CANONICAL_FP32 = 2,  /* canonical order, four FP32 FMA stages */
  CMPS_FORM_CANONICAL_TC = 3     /* canonical order, four tcgen05 split-BF16 stages */
};

typedef struct cmps_context cmps_context;
typedef struct cmps_heff cmps_heff;
typedef struct cmps_svd cmps_svd;
typedef struct cmps_block cmps_block;

/* Charge rules of the model: nq entries, the N of each Z_N charge (<=0: Z). */
typedef struct {
  int32_t nq;
  const int16_t* rules;
} cmps_charge_rules;

/* One MPX_matrix as the reference stores it (MPX_matrix.hpp:61-66).
 * charges: for index i, element e, component c:
 *   charges[(offset_i + e) * nq + c], offset_i = sum_{j<i} sizes[j].
 * Physical indices carry the basis charges like any other index. */
typedef struct {
  int32_t num_indices;
  int32_t num_row_indices;
  const uint8_t* inward;      /* [num_indices] 1 = ingoing */
  const uint8_t* physical;    /* [num_indices] */
  const int64_t* sizes;       /* [num_indices] */
  const int16_t* charges;     /* [sum(sizes) * nq] */
  int64_t rows, cols;         /* CSC matrix shape */
  const int64_t* colptr;      /* [cols + 1] */
  const int64_t* rowind;      /* [nnz] */
  const double* values;       /* [2 * nnz] interleaved complex */
} cmps_mpx_desc;

/* ---- context ---------------------------------------------------------- */
int cmps_context_create(int device, cmps_context** out);
int cmps_context_destroy(cmps_context* ctx);
/* Device memory of the library comes from the device's stream-ordered pool,
 * which keeps what is freed.  cmps_context_reserve(ctx, bytes) maps `bytes`
 * into the pool at once, so that the first steps of a run, whose buffers grow
 * with the bond dimension, do not pay for mapping new memory one allocation
 * at a time; bytes = 0 returns the pool's unused memory to the device. */
int cmps_context_reserve(cmps_context* ctx, uint64_t bytes);
const char* cmps_last_error(void);
/* Library build string (architecture, kernels compiled in). */
const char* cmps_version(void);

/* ---- effective Hamiltonian (TwoVertexComponents) ----------------------
 * Replaces the TwoVertexComponents constructor (DMRG_routines.cpp:779-833):
 * L is the 6-index left block (a' = index 1, b = index 3, a = index 5; the
 * rest size-1 dummies: MakeLeftBlock / MakeInitialLeftBlock /
 * MakeDummyLeftBlock, DMRG_routines.cpp:583-632), W the 4-index MPO
 * (sigma', b_left, sigma, b_right: make_model.hpp:613-618), R the 6-index
 * right block (a' = 0, b = 2, a = 4).  Everything is uploaded once and kept
 * on the device as charge-sector block lists; LeftPart and RightPart are
 * formed on the device. */
int cmps_heff_create(cmps_context* ctx, const cmps_charge_rules* rules,
                     const cmps_mpx_desc* L, const cmps_mpx_desc* W,
                     const cmps_mpx_desc* R, int precision, cmps_heff** out);
/* Same, with the environments taken from device-resident blocks produced by
 * cmps_heff_left_block / cmps_heff_right_block (no host round trip); the
 * blocks are copied, the caller keeps ownership. */
int cmps_heff_create_from_blocks(cmps_context* ctx, const cmps_charge_rules* rules,
                                 const cmps_block* L, const cmps_mpx_desc* W,
                                 const cmps_block* R, int precision, cmps_heff** out);
/* Upload a reference-layout block (6-index MPX_matrix, left or right) as a
 * device block, e.g. the dummy end blocks (MakeDummyLeftBlock /
 * MakeDummyRightBlock, DMRG_routines.cpp:613-653).  W gives the MPO index. */
int cmps_block_create(cmps_context* ctx, const cmps_charge_rules* rules,
                      const cmps_mpx_desc* block, const cmps_mpx_desc* W, int right,
                      cmps_block** out);
int cmps_heff_destroy(cmps_heff* h);
/* n_allowed = allowed_indices.size() (the ARPACK vector length);
 * full_length = TwoVertexComponents::length() (DMRG_routines.hpp:211). */
int cmps_heff_length(const cmps_heff* h, int64_t* n_allowed, int64_t* full_length);
/* allowed_indices in ARPACK order (DMRG_routines.cpp:808-824). */
int cmps_heff_allowed_indices(const cmps_heff* h, int64_t* out);
/* Replaces TwoVertexMPOMPSMultiply (DMRG_routines.cpp:898-974): in and out
 * are HOST arrays of n_allowed complex doubles (ARPACK's workd slices). */
int cmps_heff_apply(cmps_heff* h, const double* in, double* out);
/* Same on DEVICE arrays, stream-ordered on `stream` (cudaStream_t or NULL). */
int cmps_heff_apply_device(cmps_heff* h, const double* d_in, double* d_out, void* stream);
/* Algorithmic flops of one apply: canonical = L.theta, W1, W2, .R stages
 * over non-zero MPO entries (8 per complex MAC); executed = what the grouped
 * GEMM launches of the handle's precision and contraction order issue. */
int cmps_heff_flops(const cmps_heff* h, double* canonical, double* executed);
/* Measured tile shapes (no counterpart in the reference): every grouped GEMM
 * plan the handle's matvec runs (folded or canonical, FP64 or the FP32
 * canonical form; the tcgen05 split stages have fixed tiles) is launched
 * with each output tile shape -- 64x64, 32x128, 128x32 -- and keeps the
 * fastest.  Choices are cached per process by plan signature; `cached`
 * counts the plans that took a cached choice.  ms_heuristic / ms_best: the
 * summed per-launch times of the tuned plans with the padded-work choice and
 * with the measured one.  Outputs may be NULL. */
int cmps_heff_autotune(cmps_heff* h, int* tuned, int* cached, double* ms_heuristic, double* ms_best);
/* Chooses the contraction order of the FP64 matvec (CMPS_ORDER_*); no
 * counterpart in the reference, whose only order is the folded one. */
int cmps_heff_set_order(cmps_heff* h, int order);
/* The order in use (CMPS_ORDER_FOLDED or _CANONICAL) and the flops each
 * order executes per FP64 matvec; any output may be NULL. */
int cmps_heff_order(const cmps_heff* h, int* active, double* executed_folded, double* executed_canonical);
/* The form of the split operator the handle's precision runs (CMPS_FORM_*). */
int cmps_heff_split_form(const cmps_heff* h, int* form);
/* H_eff matvec that allocates nothing (no counterpart in the reference).
 * For callers that cannot call cudaMalloc when they apply H_eff: an
 * eigensolver callback (ARPACK's MV, called hundreds of times per step)
 * inside a host application whose device memory belongs to its own pool or
 * caching allocator, where an allocation from the callback would fail or
 * would add an allocation and a device-wide synchronisation per iteration.
 * Same inputs and result as cmps_heff_apply_device (FP64 handles only), but
 * its scratch -- the gathered vector, the stage-1 intermediate and the
 * stage-2 output, 4 * n_allowed + 2 * |T| doubles -- lives in one static
 * device array of at most 32 MiB held by every GPU that loads the library;
 * larger problems are rejected with CMPS_ERR_ARG.  The first call on a device
 * looks up that array's device address (cudaGetSymbolAddress), so make the
 * first call before any stream capture.  All calls share the array: calls
 * that overlap on the GPU race.  Nothing in it needs to start at zero. */
int cmps_heff_apply_device_noalloc(cmps_heff* h, const double* d_in, double* d_out, void* stream);
/* Excited-state projectors: TwoVertexComponents::ProjectorTensors
 * (DMRG_routines.hpp:205, built by ProjectorBlocks::makePTensor, :830).
 * count tensors P_p (each n_allowed interleaved complex in ARPACK order, the
 * layout of TwoVertexMPOMPSMultiply's vectors) with weights w_p: every
 * application of H_eff -- cmps_heff_apply[_device], the theta-layout apply and
 * the eigensolver's steps, FP64 and split-TF32 -- adds
 * sum_p w_p (P_p . x) conj(P_p), with the product P_p . x taken without
 * conjugation (DMRG_routines.cpp:947-973).  count = 0 removes them; at most
 * 64.  The adjoint (dE/dlambda) ignores them, as they do not depend on the
 * coupling; the no-allocation matvec refuses a handle that has them. */
int cmps_heff_set_projectors(cmps_heff* h, int count, const double* tensors, const double* weights);
/* Sharding the matvec by output sector (no reference counterpart: the
 * reference matvec runs on one host).  In the theta layout a vector is
 * planar -- `total` real parts, then `total` imaginary parts -- and output
 * sector m of H_eff occupies elements [offsets[m], offsets[m+1]) of each
 * plane.  Each GPU of a sharded run holds the same handle (the environments
 * and the MPO are replicated), computes the output sectors it owns from the
 * input sectors it reads, and receives those from the ranks that own them
 * (an exchange per matvec, done by the caller).
 *
 * cmps_heff_sector_table: call with offsets = flops = NULL to read the
 * sector count into *n_sectors, then with arrays of *n_sectors + 1 offsets
 * and *n_sectors flops (the executed flops of the full FP64 matvec that
 * produce output sector m, the cost model for balancing the shards). */
int cmps_heff_sector_table(const cmps_heff* h, int64_t* n_sectors, int64_t* offsets, double* flops);
/* Restrict the matvec to the output sectors with owned[m] != 0 (n_sectors
 * bytes): the GEMM plans keep only the tasks that produce them, and the
 * other output blocks are left unwritten.  A handle that does not own every
 * sector accepts only cmps_heff_apply_theta_device (the ARPACK-order apply,
 * the eigensolver, the adjoint and the stage timing return CMPS_ERR_STATE);
 * owning every sector again restores them.  It also returns the vector
 * windows to the theta layout. */
int cmps_heff_set_owned(cmps_heff* h, const uint8_t* owned);
/* The input sectors the owned output sectors read (n_sectors bytes, 1 =
 * read), for the current owned set and contraction order. */
int cmps_heff_input_sectors(const cmps_heff* h, uint8_t* needed);
/* Vector windows, so that a rank holds only what it reads and writes: input
 * sector m (each sector the owned outputs read) is at in_base[m] of an input
 * of in_len entries per plane, owned output sector m at out_base[m] of an
 * output of out_len entries per plane (n_sectors entries each; other entries
 * are ignored).  Every such sector must lie inside its window.  The plans are
 * rebuilt; refused while projectors are set. */
int cmps_heff_set_windows(cmps_heff* h, const int64_t* in_base, int64_t in_len, const int64_t* out_base,
                          int64_t out_len);
/* theta-layout matvec on DEVICE arrays, stream-ordered: d_in holds the input
 * (2 * in_len doubles, planar; the whole vector, 2 * total, unless windows
 * are set), d_out receives the owned output sectors (2 * out_len doubles;
 * d_out != d_in). */
int cmps_heff_apply_theta_device(cmps_heff* h, const double* d_in, double* d_out, void* stream);
/* ARPACK order (n_allowed interleaved complex) <-> theta layout, on DEVICE
 * arrays.  theta_to_arpack reads every sector of its input. */
int cmps_heff_theta_from_arpack(cmps_heff* h, const double* d_arpack, double* d_theta, void* stream);
int cmps_heff_theta_to_arpack(cmps_heff* h, const double* d_theta, double* d_arpack, void* stream);
/* Stage timing for roofline accounting: runs `reps` device applies on
 * `stream` (cudaStream_t or NULL) and returns the average duration in ms of
 * each launch, measured with CUDA events on that stream:
 * ms[0] gather (ARPACK order -> sector blocks), ms[1] stage-1 grouped GEMM,
 * ms[2] stage-2 grouped GEMM, ms[3] scatter. */
int cmps_heff_time_stages(cmps_heff* h, const double* d_in, double* d_out, void* stream,
                          int reps, double* ms);
/* Synchronises the handle's stream and reports any failure the device
 * kernels recorded asynchronously (a bounded tcgen05 pipeline wait that
 * timed out); CMPS_OK otherwise. */
int cmps_heff_status(cmps_heff* h);
/* Switch the contraction arithmetic of an existing handle (CMPS_FP64 or
 * CMPS_SPLIT_TF32). */
int cmps_heff_set_precision(cmps_heff* h, int precision);

/* Lowest eigenpair (smallest real part) of H_eff, device Lanczos in FP64
 * with full re-orthogonalisation and explicit restarts.  Replaces
 * TwoVertexComponents::HED -> arpack::arpack_eigs (DMRG_routines.cpp:835-896,
 * arpack_interface.hpp:174-237); the eigenvector is post-processed as HED
 * does: phase of the largest entry removed, entries <= eps*max dropped,
 * FixComplexPrecision.  guess: host, n_allowed complex, or NULL.  evec:
 * host, n_allowed complex, or NULL (the vector stays on the device for
 * cmps_heff_theta_svd either way).  tol: residual norm / |eigenvalue|. */
int cmps_heff_eigs(cmps_heff* h, const double* guess, double tol, int max_restarts,
                   int krylov_dim, double* eval, double* evec, int* matvecs);
/* Work of the last cmps_heff_eigs call on this handle (no reference
 * counterpart; diagnostics).  With CMPS_SPLIT_TF32 each restart cycle opens
 * with one FP64 matvec and continues with split-TF32 ones; with CMPS_FP64
 * every matvec is FP64.  ms3 = device time of {split matvecs, FP64 matvecs,
 * whole solve} (CUDA events).  Any output pointer may be NULL. */
int cmps_heff_eigs_stats(const cmps_heff* h, int* split_matvecs, int* fp64_matvecs, int* cycles, double* ms3);

/* ---- charge-block SVD of the two-vertex wavefunction ------------------
 * Replaces TwoVertexSVD -> MPX_matrix::SVD -> SparseMatrix::SVD
 * (DMRG_routines.hpp:225, MPX_matrix.cpp:157-192,
 * sparse_interface.cpp:1248-1406) for the eigenvector last produced by
 * cmps_heff_eigs (or loaded with cmps_heff_set_theta).  Truncation rule of
 * the reference: keep min(chi, total); drop the smallest values while their
 * squared sum stays below max_trunc; extend over values within 1e-3 relative
 * of the last kept one. */
int cmps_heff_set_theta(cmps_heff* h, const double* theta);
int cmps_heff_theta_svd(cmps_heff* h, int64_t chi, double max_trunc, cmps_svd** out);
int cmps_svd_destroy(cmps_svd* s);
/* kept values (descending), discarded weight, sizes of the U and V^dagger
 * CSC matrices in the reference layout (U: rows = (sigma1, a0), V^dagger:
 * cols = (sigma2, a2)). */
int cmps_svd_info(const cmps_svd* s, int64_t* kept, double* discarded_weight,
                  int64_t* nnz_u, int64_t* nnz_vd);
/* How the non-empty charge sectors were factored (a diagnostic; the result
 * does not depend on it beyond rounding): one-sided Jacobi SVD, eigenpairs
 * of the Gram matrix, or the randomized range finder (sectors much larger
 * than the bond dimension, accepted only where its leading triplets settle
 * the truncation of the whole spectrum). */
int cmps_svd_routes(const cmps_svd* s, int* n_exact, int* n_gram, int* n_randomized);
/* values[kept]; new bond charges[kept * nq]; U and V^dagger in CSC. */
int cmps_svd_copy(const cmps_svd* s, double* values, int16_t* new_charges,
                  int64_t* u_colptr, int64_t* u_rowind, double* u_values,
                  int64_t* vd_colptr, int64_t* vd_rowind, double* vd_values);

/* ---- environment updates ---------------------------------------------
 * New left block L' = A^dagger (W (L A)) from the handle's L and W and the
 * U of `s` (MakeLeftBlock, DMRG_routines.cpp:594-602); new right block
 * R' = B^dagger (W (R B)) from V^dagger of `s` (MakeRightBlock, :603-611).
 * The result stays on the device; cmps_block_info / cmps_block_copy export
 * it as the reference's 6-index MPX_matrix (rows = a', cols = (b, a)). */
int cmps_heff_left_block(cmps_heff* h, const cmps_svd* s, cmps_block** out);
int cmps_heff_right_block(cmps_heff* h, const cmps_svd* s, cmps_block** out);
int cmps_block_destroy(cmps_block* b);
int cmps_block_info(const cmps_block* b, int64_t* chi, int64_t* mpo_dim, int64_t* nnz);
/* a_charges[chi * nq] (the new bond), CSC of the (chi) x (mpo_dim * chi)
 * matrix: row = a', col = b + mpo_dim * a. */
int cmps_block_copy(const cmps_block* b, int16_t* a_charges, int64_t* colptr,
                    int64_t* rowind, double* values);

/* ---- adjoint of the H_eff contraction (no reference counterpart) -------
 * Derivative of the variational energy E = <theta|H_eff|theta>/<theta|theta>
 * with respect to one coupling lambda of the vertex MPO, W = W0 + lambda dW
 * (an interchain coupling, a field).  theta is the wavefunction last produced
 * by cmps_heff_eigs (or set by cmps_heff_set_theta).  dW has the MPO's
 * indices and charges; its non-zero entries must lie inside the non-zero
 * pattern of W (evaluate at a non-zero coupling).  dL / dR are the
 * environments' own derivatives (dW inserted at one earlier vertex; layout of
 * the handle's L / R), or NULL for zero.  grad = Re <theta|dH_eff|theta> /
 * <theta|theta>, contracted in FP64 through the matvec's own grouped-GEMM
 * plans (two matvecs). */
int cmps_heff_adjoint(cmps_heff* h, const cmps_mpx_desc* dW, const cmps_block* dL,
                      const cmps_block* dR, double* grad);

/* ---- device-resident iDMRG growth (SuperBlock) -------------------------
 * Replaces SuperBlock::grow_two_vertex (DMRG_routines.cpp:346-374) with
 * everything on the device: the new environments come from the previous
 * step's H_eff and SVD (MakeLeftBlock / MakeRightBlock), the start vector
 * from the device form of MakePrediction (:693-707), then the ground state
 * (cmps_heff_eigs) and the truncated SVD.  The first call solves the two
 * vertex problem on the dummy end blocks (MakeDummyLeftBlock /
 * MakeDummyRightBlock, :613-653), as SuperBlock::initialise does (:309-344).
 * target: the target charges (nq values, NULL = all zero). */
typedef struct cmps_dmrg cmps_dmrg;
int cmps_dmrg_create(cmps_context* ctx, const cmps_charge_rules* rules, const cmps_mpx_desc* W,
                     const int16_t* target, int precision, cmps_dmrg** out);
int cmps_dmrg_destroy(cmps_dmrg* d);
int cmps_dmrg_set_solver(cmps_dmrg* d, double tol, int max_restarts, int krylov_dim);
/* One growth step.  row5 = {energy, energy / vertices, entropy, truncation,
 * fidelity} -- the Data row of iDMRG_DRV's energies file (fidelity =
 * CheckConvergence, DMRG_routines.cpp:769-771, on by default; NaN when
 * turned off with cmps_dmrg_set_fidelity(d, 0)); bond_dim = kept states;
 * matvecs = H_eff applications; ms4 = device time of {environment update +
 * H_eff build + prediction, eigensolve, SVD (+ fidelity), total} in ms (CUDA
 * events).  Any output pointer but row5 may be NULL. */
int cmps_dmrg_grow(cmps_dmrg* d, int64_t chi, double max_trunc, double* row5, int64_t* bond_dim,
                   int* matvecs, double* ms4);
/* The current (rescaled) singular values, bond_dim of them, descending. */
int cmps_dmrg_values(const cmps_dmrg* d, double* values);
/* The translation-invariant unit cell of the last growth step and its
 * energy per vertex: what iDMRG_DRV measures after every step
 * (iDMRG_DRV.cpp:71-77), Orthogonalise(MPSDecomposition, PreviousLambda)
 * (measurement.cpp:180-246, 254-257) followed by
 * iTwoVertexEnergy(ColX, RowX, H1, UnitCell) (measurement.cpp:378-397),
 * with H1, ColX and RowX the on-vertex, column and row blocks of the
 * handle's MPO (measurement.cpp:371-376).  The cell is U and
 * diag(s) V^dagger diag(1/lambda_prev) (UnitCell.hpp:42-47); the dominant
 * left and right eigenpairs of its transfer matrix come from a restarted
 * Arnoldi iteration to residual <= tol * |eigenvalue| (Krylov dimension
 * krylov_dim, at most 64).  out6 = {energy per vertex, entropy of the
 * orthogonalised boundary values, left and right dominant eigenvalues,
 * number of boundary values (those whose square is above 1e-14 of the
 * largest), imaginary part of the energy}.  Needs two growth steps or more
 * (lambda_prev must live on the cell's end bonds; the reference measures
 * after its two warm-up steps, iDMRG_DRV.cpp:46-50,64-71); CMPS_ERR_SOLVER
 * where Orthogonalise returns an empty cell (complex dominant eigenvalue,
 * SqrtDR with eigenvalues of both signs). */
int cmps_dmrg_unit_cell(cmps_dmrg* d, double tol, int krylov_dim, double* out6);
/* ---- finite sweeps (FiniteDMRG, fDMRG_routines.cpp:19-66) ---------------
 * cmps_dmrg_keep_blocks(d, 1) before the first growth step keeps the left
 * and right blocks of every length (BlocksStructure, kept in device memory
 * instead of the reference's .BLOCK files).  After growth to the chain
 * length, cmps_dmrg_move(d, +1 / -1, ...) is move_right_two_vertex /
 * move_left_two_vertex (DMRG_routines.cpp:376-444): the block of the side
 * the window leaves is updated with this window's U or V^dagger, the new
 * window is solved and truncated (no weight cut next to an end), and row5 is
 * the reference's energies row (fidelity NaN).  The start vector of a sweep
 * step is MakeRFinitePrediction / MakeLFinitePrediction (:709-716): this
 * window's Lambda V^dagger (U Lambda) times the stored right (left) MPS
 * tensor of the vertex entering the window.  cmps_dmrg_position
 * returns the number of vertices left of the window and the chain length. */
int cmps_dmrg_keep_blocks(cmps_dmrg* d, int keep);
int cmps_dmrg_set_fidelity(cmps_dmrg* d, int on);
/* Contraction order of every later step's H_eff (CMPS_ORDER_*, default
 * AUTO; see cmps_heff_set_order).  No counterpart in the reference. */
int cmps_dmrg_set_order(cmps_dmrg* d, int order);
/* Autotune (cmps_heff_autotune) every later step's H_eff; the stats are
 * summed over the run. */
int cmps_dmrg_set_autotune(cmps_dmrg* d, int on);
int cmps_dmrg_autotune_stats(const cmps_dmrg* d, int* tuned, int* cached, double* ms_heuristic, double* ms_best);
int cmps_dmrg_move(cmps_dmrg* d, int direction, int64_t chi, double max_trunc, double* row5,
                   int64_t* bond_dim, int* matvecs, double* ms4);
int cmps_dmrg_position(const cmps_dmrg* d, int64_t* nleft, int64_t* size);

/* ---- excited states (fDMRG_DRV -X, ExcitedStateFiniteDMRG,
 * fDMRG_routines.cpp:68-244; ProjectorBlocks, DMRG_routines.cpp:446-581) ----
 * cmps_dmrg_project_state(d, w) stores the current state of a finite chain
 * (its left tensors, the window's U diag(lambda) and V^dagger, its right
 * tensors; on the device) as a state to project out with weight w
 * (next_state, fDMRG_routines.hpp:39-44; the reference's default weight is
 * 100).  Every later step builds, on the device, the overlaps of each stored
 * state with the current left and right bases and its projector tensor P on
 * the new window, and solves H_eff + sum_p w_p |P_p*><P_p*| (the projector
 * term of TwoVertexMPOMPSMultiply, DMRG_routines.cpp:947-973) with no
 * prediction vector, as the reference's excited sweeps do.  Growth steps are
 * refused while states are stored.  cmps_dmrg_solve solves the current window
 * again with its environments, without moving (ExcitedStateFiniteDMRG::init),
 * and returns the same row as cmps_dmrg_move.  cmps_dmrg_projector copies the
 * current window's P of stored state `index` in ARPACK order (n_allowed
 * interleaved complex values). */
int cmps_dmrg_project_state(cmps_dmrg* d, double weight);
int cmps_dmrg_projected_states(const cmps_dmrg* d, int* count);
int cmps_dmrg_solve(cmps_dmrg* d, int64_t chi, double max_trunc, double* row5, int64_t* bond_dim, int* matvecs,
                    double* ms4);
int cmps_dmrg_projector(const cmps_dmrg* d, int index, double* arpack_out);
/* Allowed entries and full length of the current window (the length of a
 * vector in ARPACK order, TwoVertexComponents::length()). */
int cmps_dmrg_window_length(const cmps_dmrg* d, int64_t* n_allowed, int64_t* full_length);

/* Coupling gradient along the growth (no reference counterpart).  Set before
 * the first growth step: dW as for cmps_heff_adjoint (NULL turns it off).
 * Each step then carries the derivative environments dL, dR (the environment
 * update with LeftPart / RightPart replaced by their derivatives, the step's
 * truncation factors held fixed) and cmps_dmrg_gradient returns dE/dlambda of
 * the last step's energy (cmps_heff_adjoint with those environments). */
int cmps_dmrg_set_gradient(cmps_dmrg* d, const cmps_mpx_desc* dW);
int cmps_dmrg_gradient(const cmps_dmrg* d, double* grad);
/* Breakdown of the last growth step (no reference counterpart;
 * diagnostics).  Writes the first n (<= 21) of: {environment update ms, H_eff
 * build + prediction ms, eigensolve ms, SVD ms, total ms (device time, CUDA
 * events); split matvecs, FP64 matvecs, restart cycles, split matvec ms,
 * FP64 matvec ms; host wall ms of environment update, H_eff build, split
 * operand preparation, prediction, release of the previous step, SVD, whole
 * step; SVD sectors factored exactly, by the Gram matrix, by the randomized
 * route; contraction order of the FP64 matvec (CMPS_ORDER_*)}. */
int cmps_dmrg_profile(const cmps_dmrg* d, double* out, int n);

/* ---- MPX_matrix files (host only) ---------------------------------------
 * The reference's binary MPX_matrix format: MPX_matrix::store /
 * load_MPX_matrix_binary (MPX_matrix.cpp:219-247,593-607, MPXIndex.cpp:8-23,
 * 98-121, states.cpp:59-61, sparse_interface.cpp:727-835).  It carries the
 * .BLOCK environment checkpoints (BlocksStructure::save_left_block etc.,
 * DMRG_routines.cpp:65-186) and the .MPS_matrix / .MPX_matrix state files.
 * These entry points touch no device memory and need no GPU.
 *
 * Store m (nq charges per state) to path, as MPX_matrix::store writes it;
 * a physical index is written without its charges. */
int cmps_mpx_store(const cmps_mpx_desc* m, int32_t nq, const char* path);
/* Sizes of a stored MPX_matrix: index count, row-index count, total index
 * elements (sum of the index sizes), CSC shape and number of entries. */
int cmps_mpx_stat(const char* path, int32_t nq, int32_t* num_indices, int32_t* num_row_indices,
                  int64_t* total_elements, int64_t* rows, int64_t* cols, int64_t* nnz);
/* Read a stored MPX_matrix into caller buffers sized from cmps_mpx_stat:
 * inward / physical / sizes [num_indices], charges [total_elements * nq],
 * colptr [cols + 1], rowind [nnz], values [2 * nnz] interleaved complex.
 * Physical indices take basis_charges [basis_size * nq] (the model's
 * spectrum, as load_MPXIndex_binary does); their stored size must equal
 * basis_size.  Of the nzmax entries stored, the first colptr[cols] are kept
 * (load_SparseMatrix_binary). */
int cmps_mpx_load(const char* path, int32_t nq, const int16_t* basis_charges, int64_t basis_size,
                  uint8_t* inward, uint8_t* physical, int64_t* sizes, int16_t* charges,
                  int64_t* colptr, int64_t* rowind, double* values);

#ifdef __cplusplus
}
#endif
#endif /* CHAINAMPS_B200_H */
