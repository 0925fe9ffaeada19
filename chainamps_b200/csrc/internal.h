// Internal declarations of the chainamps_b200 library (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <array>
#include <functional>
#include <map>
#include <string>
#include <vector>

#include "chainamps_b200.h"

namespace cmps {

constexpr int kMaxQ = 4;  // charges per state (QuantumNumberInt each)
using QKey = std::array<int16_t, kMaxQ>;

// Error reporting: thread-local last-error string, returned codes.
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);

#define CMPS_CUDA(call)                                                              \
  do {                                                                               \
    cudaError_t _e = (call);                                                         \
    if (_e != cudaSuccess)                                                           \
      return ::cmps::fail(CMPS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
  } while (0)

#define CMPS_TRY(call)            \
  do {                            \
    int _s = (call);              \
    if (_s != CMPS_OK) return _s; \
  } while (0)

// Copies and fills outside the matvec.  The library's streams are created
// non-blocking, so the legacy default stream (plain cudaMemcpy / cudaMemset)
// is not ordered with them: a fill could land after the kernels that write the
// buffer, an upload after the kernels that read it.  These issue the copy on
// the stream the neighbouring kernels use and wait for it before returning.
int copy_wait(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind, cudaStream_t st);
int zero_wait(void* dst, size_t bytes, cudaStream_t st);

// Device memory of the library.  A DMRG step frees and re-allocates buffers
// of several GB (Krylov basis, LeftPart/RightPart, T, split operands, SVD
// work); plain cudaMalloc / cudaFree map and unmap that memory every step,
// which costs up to hundreds of ms at unpredictable points.  These take it
// from the current device's stream-ordered pool instead, whose release
// threshold is raised so freed memory stays mapped for the next step.  Both
// keep the synchronisation of cudaMalloc / cudaFree: dmalloc returns memory
// usable from any stream, dfree waits for the device before releasing.
cudaError_t dmalloc(void** p, size_t bytes);
cudaError_t dfree(void* p);

template <class T>
inline cudaError_t dmalloc(T** p, size_t bytes) {
  return dmalloc(reinterpret_cast<void**>(p), bytes);
}

// Dynamic shared memory opt-in of a kernel above 48 KB.  cudaFuncSetAttribute
// applies to the current device only, so the opt-in is made once per (kernel,
// device ordinal), under a lock: a process may drive several GPUs, and the
// SVD's worker threads launch the same kernels concurrently.
int ensure_smem_optin(const void* func, int bytes);

// Charge arithmetic of State (states.hpp:176-206).
struct Rules {
  int nq = 0;
  int16_t n[kMaxQ] = {0, 0, 0, 0};
  QKey add(const QKey& a, const QKey& b) const;
  QKey sub(const QKey& a, const QKey& b) const;
  QKey zero() const { return QKey{0, 0, 0, 0}; }
};

// Elements of one bond index grouped by charge.  Element order is the
// reference's element order; sectors are numbered by first appearance.
struct Bond {
  std::vector<QKey> sq;                     // charge of each sector
  std::vector<int64_t> sdim;                // elements per sector
  std::vector<int32_t> esec;                // element -> sector
  std::vector<int64_t> epos;                // element -> position inside its sector
  std::vector<std::vector<int64_t>> selem;  // sector -> elements in order
  std::map<QKey, int> lookup;
  int64_t size() const { return (int64_t)esec.size(); }
  int nsec() const { return (int)sq.size(); }
  int find(const QKey& q) const {
    auto it = lookup.find(q);
    return it == lookup.end() ? -1 : it->second;
  }
  void build(const std::vector<QKey>& charges);
  std::vector<QKey> element_charges() const;
};

// A split-precision form (the mixed eigensolver's low-precision operator).
inline bool is_split(int precision) { return precision == CMPS_SPLIT_TF32 || precision == CMPS_SPLIT_BF16; }

// Device buffer of complex values stored as two planes (re then im).
struct Planar {
  double* d = nullptr;
  int64_t len = 0;  // complex elements
  double* re() const { return d; }
  double* im() const { return d + len; }
  int alloc(int64_t n);
  void release();
};

// Single-precision counterpart of Planar (re plane, then im plane).  A view
// into another allocation (owned = false) is not freed by release().
struct Planar32 {
  float* d = nullptr;
  int64_t len = 0;
  bool owned = false;
  float* re() const { return d; }
  float* im() const { return d + len; }
  int alloc(int64_t n);
  void release();
};

// An environment (left or right block) on the device.  Block (b, s) of a
// left block is the dense [a', a] matrix L^b restricted to a-sector s and
// a'-sector s' = sector(q_s + q_b), row-major (dim s') x (dim s).  A right
// block stores R^b transposed: [a, a'], (dim t) x (dim t').
struct Env {
  Bond a;
  int D = 0;
  std::vector<QKey> bq;         // MPO bond charges
  std::vector<int64_t> off;     // D * nsec, -1 if the block is absent
  std::vector<int32_t> partner; // D * nsec: s' (the a' sector) or -1
  Planar data;
  bool right = false;
  int64_t block_rows(int b, int s) const;
  int64_t block_cols(int b, int s) const;
};

struct WEntry {
  int sp, bl, s, br;
  double wr, wi;
};

// Grouped complex GEMM work description (device arrays).
// With n_in > 0 the N index is two-level: column n of C (and of B) lies at
// (n / n_in) * ldc_out + n % n_in (B: * ldb_out) from the row start, i.e. N
// runs over n / n_in blocks of n_in consecutive elements; the plan must set
// GemmPlan::nsplit.
struct GemmTask {
  int64_t c_off;
  int32_t m, n, ldc;
  int32_t t0, t1;  // term range
  int32_t n_in;    // 0: plain N
  int32_t ldc_out, pad;
};
struct GemmTerm {
  int64_t a_off, b_off;
  int32_t k, lda, ldb, ldb_out;
};
struct GemmTile {
  int32_t task, m0, n0, pad;
};

struct GemmPlan {
  std::vector<GemmTask> tasks;
  std::vector<GemmTerm> terms;
  std::vector<GemmTile> tiles;
  GemmTask* d_tasks = nullptr;
  GemmTerm* d_terms = nullptr;
  GemmTile* d_tiles = nullptr;
  double flops = 0.0;
  bool nsplit = false;  // tasks use the two-level N index (n_in > 0)
  int shape = -1;       // output tile shape (gemm_shape_m / _n), chosen by upload
  // Picks the tile shape for these tasks, splits them into tiles and copies
  // the plan to the device.
  int upload(cudaStream_t st);
  // The tiles again for another shape (an uploaded plan; tasks and terms unchanged).
  int retile(int shape, cudaStream_t st);
  // Host check, before any launch, that every operand and output range lies
  // inside its buffer (lengths in complex elements).
  int validate(bool a_h, bool b_h, int64_t a_len, int64_t b_len, int64_t c_len, const char* what) const;
  void release();
};

// Empirical tile-shape choice: `run` launches the plan once; every shape is
// timed (one warm-up, three timed launches, CUDA events on st) and the
// fastest kept.  Results are cached per process by plan signature (role,
// task and term counts, flops, padded-work choice), so a plan of the same
// population is not timed again.
struct TuneStats {
  int tuned = 0, cached = 0;
  double ms_heuristic = 0.0, ms_best = 0.0;  // per launch, summed over the tuned plans
};
int autotune_plan(GemmPlan& p, int role, const std::function<int()>& run, cudaStream_t st, TuneStats* stats);

// Block AXPY lists: dst block = sum_t w_t * src_t (same shapes).
struct AxpyBlock {
  int64_t dst_off, len;
  int32_t t0, t1;
};
struct AxpyTerm {
  int64_t src_off;
  double wr, wi;
};

// ---- kernels (launchers) ---------------------------------------------------
// output tile shapes of zgemm_grouped_fp64 (GemmPlan::shape)
int gemm_shape_m(int shape);
int gemm_shape_n(int shape);
int launch_zgemm_fp64(const GemmPlan& p, bool a_h, bool b_h, const Planar& A, const Planar& B,
                      Planar& C, cudaStream_t st);
// FP32 grouped complex GEMM (cgemm_fp32.cu): the same plans as
// launch_zgemm_fp64 without conjugated operands.
int launch_cgemm_fp32(const GemmPlan& p, const Planar32& A, const Planar32& B, Planar32& C, cudaStream_t st);
int to_fp32(const double* re, const double* im, int64_t n, Planar32& out, cudaStream_t st);
int to_fp64(const Planar32& in, int64_t n, double* re, double* im, cudaStream_t st);
int launch_block_axpy(const AxpyBlock* d_blocks, int nblocks, const AxpyTerm* d_terms,
                      const Planar& src, Planar& dst, cudaStream_t st, bool accumulate = false);

}  // namespace cmps
