// C ABI entry points (include/chainamps_b200.h): argument checking, error
// strings, context and handle lifetime.  No entry point aborts; every
// failure is an int status plus cmps_last_error().
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <set>
#include <string>
#include <utility>

#include "heff.h"

namespace cmps {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
int fail(int code, const std::string& msg) {
  set_error(msg);
  return code;
}

int copy_wait(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind, cudaStream_t st) {
  if (!bytes) return CMPS_OK;
  CMPS_CUDA(cudaMemcpyAsync(dst, src, bytes, kind, st));
  CMPS_CUDA(cudaStreamSynchronize(st));
  return CMPS_OK;
}

static std::mutex g_pool_mu;
static bool g_pool_ready[64] = {false};

static cudaError_t pool_setup(int dev) {
  if (dev < 0 || dev >= 64) return cudaSuccess;  // beyond the table: default pool settings
  std::lock_guard<std::mutex> lock(g_pool_mu);
  if (g_pool_ready[dev]) return cudaSuccess;
  cudaMemPool_t pool;
  cudaError_t e = cudaDeviceGetDefaultMemPool(&pool, dev);
  if (e != cudaSuccess) return e;
  uint64_t keep = UINT64_MAX;
  e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  if (e == cudaSuccess) g_pool_ready[dev] = true;
  return e;
}

cudaError_t dmalloc(void** p, size_t bytes) {
  *p = nullptr;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = pool_setup(dev);
  if (e == cudaSuccess) e = cudaMallocAsync(p, std::max<size_t>(bytes, 1), cudaStreamLegacy);
  if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamLegacy);
  return e;
}

cudaError_t dfree(void* p) {
  if (!p) return cudaSuccess;
  cudaError_t e = cudaDeviceSynchronize();
  cudaError_t f = cudaFreeAsync(p, cudaStreamLegacy);
  return e != cudaSuccess ? e : f;
}

static std::mutex g_optin_mu;
static std::set<std::pair<const void*, int>> g_optin_done;  // (kernel, device)

int ensure_smem_optin(const void* func, int bytes) {
  int dev = 0;
  CMPS_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(g_optin_mu);
  if (g_optin_done.count({func, dev})) return CMPS_OK;
  CMPS_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  g_optin_done.insert({func, dev});
  return CMPS_OK;
}

int zero_wait(void* dst, size_t bytes, cudaStream_t st) {
  if (!bytes) return CMPS_OK;
  CMPS_CUDA(cudaMemsetAsync(dst, 0, bytes, st));
  CMPS_CUDA(cudaStreamSynchronize(st));
  return CMPS_OK;
}

static int rules_from(const cmps_charge_rules* cr, Rules& r) {
  if (!cr || cr->nq < 1 || cr->nq > kMaxQ || !cr->rules)
    return fail(CMPS_ERR_ARG, "charge rules: need 1.." + std::to_string(kMaxQ) + " charges");
  r.nq = cr->nq;
  for (int i = 0; i < kMaxQ; ++i) r.n[i] = i < cr->nq ? cr->rules[i] : 0;
  return CMPS_OK;
}

static int use_device(cmps_context* ctx) {
  if (!ctx) return fail(CMPS_ERR_ARG, "null context");
  CMPS_CUDA(cudaSetDevice(ctx->device));
  cudaGetLastError();  // drop a stale non-sticky error of an unrelated earlier call
  return CMPS_OK;
}

}  // namespace cmps

using namespace cmps;

extern "C" {

const char* cmps_last_error(void) { return g_last_error.c_str(); }

const char* cmps_version(void) {
  return "chainamps_b200 1.0 sm_100a: fp64 DMMA grouped zgemm, device Lanczos, cusolver block SVD";
}

int cmps_context_create(int device, cmps_context** out) {
  if (!out) return fail(CMPS_ERR_ARG, "null output pointer");
  *out = nullptr;
  int n = 0;
  CMPS_CUDA(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n) return fail(CMPS_ERR_ARG, "no such CUDA device");
  CMPS_CUDA(cudaSetDevice(device));
  auto* c = new (std::nothrow) cmps_context();
  if (!c) return fail(CMPS_ERR_NOMEM, "host allocation failed");
  c->device = device;
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return fail(CMPS_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
  }
  *out = c;
  return CMPS_OK;
}

int cmps_context_reserve(cmps_context* ctx, uint64_t bytes) {
  if (!ctx) return fail(CMPS_ERR_ARG, "null context");
  CMPS_CUDA(cudaSetDevice(ctx->device));
  CMPS_CUDA(pool_setup(ctx->device));
  cudaMemPool_t pool;
  CMPS_CUDA(cudaDeviceGetDefaultMemPool(&pool, ctx->device));
  CMPS_CUDA(cudaDeviceSynchronize());
  if (bytes == 0) {
    CMPS_CUDA(cudaMemPoolTrimTo(pool, 0));
    return CMPS_OK;
  }
  // one allocation of the whole size maps it into the pool; freed, it stays
  // there (release threshold: keep everything) for later allocations
  void* p = nullptr;
  cudaError_t e = cudaMallocAsync(&p, (size_t)bytes, cudaStreamLegacy);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(CMPS_ERR_NOMEM, std::string("pool reservation failed: ") + cudaGetErrorString(e));
  }
  CMPS_CUDA(cudaFreeAsync(p, cudaStreamLegacy));
  CMPS_CUDA(cudaStreamSynchronize(cudaStreamLegacy));
  return CMPS_OK;
}

int cmps_context_destroy(cmps_context* ctx) {
  if (!ctx) return CMPS_OK;
  cudaSetDevice(ctx->device);
  release_solver(ctx);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return CMPS_OK;
}

int cmps_heff_create(cmps_context* ctx, const cmps_charge_rules* rules, const cmps_mpx_desc* L,
                     const cmps_mpx_desc* W, const cmps_mpx_desc* R, int precision, cmps_heff** out) {
  if (!out) return fail(CMPS_ERR_ARG, "null output pointer");
  *out = nullptr;
  CMPS_TRY(use_device(ctx));
  Rules r;
  CMPS_TRY(rules_from(rules, r));
  if (precision != CMPS_FP64 && !is_split(precision)) return fail(CMPS_ERR_ARG, "unknown precision");
  auto h = std::unique_ptr<cmps_heff>(new (std::nothrow) cmps_heff());
  if (!h) return fail(CMPS_ERR_NOMEM, "host allocation failed");
  h->impl.reset(new (std::nothrow) Heff());
  if (!h->impl) return fail(CMPS_ERR_NOMEM, "host allocation failed");
  CMPS_TRY(h->impl->build(ctx, r, L, W, R));
  CMPS_TRY(cmps_heff_set_precision(h.get(), precision));
  *out = h.release();
  return CMPS_OK;
}

int cmps_heff_create_from_blocks(cmps_context* ctx, const cmps_charge_rules* rules, const cmps_block* L,
                                 const cmps_mpx_desc* W, const cmps_block* R, int precision, cmps_heff** out) {
  if (!out || !L || !R) return fail(CMPS_ERR_ARG, "null argument");
  *out = nullptr;
  CMPS_TRY(use_device(ctx));
  Rules r;
  CMPS_TRY(rules_from(rules, r));
  if (precision != CMPS_FP64 && !is_split(precision)) return fail(CMPS_ERR_ARG, "unknown precision");
  auto h = std::unique_ptr<cmps_heff>(new (std::nothrow) cmps_heff());
  if (!h) return fail(CMPS_ERR_NOMEM, "host allocation failed");
  h->impl.reset(new (std::nothrow) Heff());
  if (!h->impl) return fail(CMPS_ERR_NOMEM, "host allocation failed");
  CMPS_TRY(h->impl->build_from_envs(ctx, r, L->env, W, R->env));
  CMPS_TRY(cmps_heff_set_precision(h.get(), precision));
  *out = h.release();
  return CMPS_OK;
}

int cmps_block_create(cmps_context* ctx, const cmps_charge_rules* rules, const cmps_mpx_desc* block,
                      const cmps_mpx_desc* W, int right, cmps_block** out) {
  if (!out || !block || !W) return fail(CMPS_ERR_ARG, "null argument");
  *out = nullptr;
  CMPS_TRY(use_device(ctx));
  Rules r;
  CMPS_TRY(rules_from(rules, r));
  Heff tmp;
  tmp.rules = r;
  CMPS_TRY(tmp.parse_mpo(W));
  auto b = std::unique_ptr<cmps_block>(new (std::nothrow) cmps_block());
  if (!b) return fail(CMPS_ERR_NOMEM, "host allocation failed");
  b->rules = r;
  CMPS_TRY(build_env_from_desc(r, block, right != 0, b->env, tmp.D, tmp.bq, ctx->stream));
  *out = b.release();
  return CMPS_OK;
}

int cmps_heff_destroy(cmps_heff* h) {
  if (!h) return CMPS_OK;
  if (h->impl) cudaSetDevice(h->impl->device);
  delete h;
  cudaGetLastError();
  return CMPS_OK;
}

int cmps_heff_length(const cmps_heff* h, int64_t* n_allowed, int64_t* full_length) {
  if (!h || !h->impl) return fail(CMPS_ERR_ARG, "null handle");
  if (n_allowed) *n_allowed = h->impl->n_allowed;
  if (full_length) *full_length = h->impl->full_length;
  return CMPS_OK;
}

int cmps_heff_allowed_indices(const cmps_heff* h, int64_t* out) {
  if (!h || !h->impl || !out) return fail(CMPS_ERR_ARG, "null argument");
  CMPS_TRY(use_device(h->impl->ctx));
  return h->impl->allowed_indices(out);
}

int cmps_heff_apply(cmps_heff* h, const double* in, double* out) {
  if (!h || !h->impl || !in || !out) return fail(CMPS_ERR_ARG, "null argument");
  CMPS_TRY(use_device(h->impl->ctx));
  return h->impl->apply_host(in, out);
}

int cmps_heff_apply_device(cmps_heff* h, const double* d_in, double* d_out, void* stream) {
  if (!h || !h->impl || !d_in || !d_out) return fail(CMPS_ERR_ARG, "null argument");
  CMPS_TRY(use_device(h->impl->ctx));
  cudaStream_t st = stream ? (cudaStream_t)stream : h->impl->ctx->stream;
  return h->impl->apply_device(d_in, d_out, st);
}

int cmps_heff_sector_table(const cmps_heff* h, int64_t* n_sectors, int64_t* offsets, double* flops) {
  if (!h || !h->impl || !n_sectors) return fail(CMPS_ERR_ARG, "null argument");
  const Heff& H = *h->impl;
  const int64_t nm = (int64_t)H.th.mq.size();
  if (offsets || flops) {
    if (*n_sectors != nm) return fail(CMPS_ERR_ARG, "sector table: *n_sectors differs from the sector count");
    if (offsets) {
      for (int64_t m = 0; m < nm; ++m) offsets[m] = H.th.base[m];
      offsets[nm] = H.th.total;
    }
    if (flops)
      for (int64_t m = 0; m < nm; ++m) flops[m] = (int64_t)H.sector_flops.size() == nm ? H.sector_flops[m] : 0.0;
  }
  *n_sectors = nm;
  return CMPS_OK;
}

int cmps_heff_set_owned(cmps_heff* h, const uint8_t* owned) {
  if (!h || !h->impl || !owned) return fail(CMPS_ERR_ARG, "null argument");
  CMPS_TRY(use_device(h->impl->ctx));
  return h->impl->set_owned(owned);
}

int cmps_heff_autotune(cmps_heff* h, int* tuned, int* cached, double* ms_heuristic, double* ms_best) {
  if (!h || !h->impl) return fail(CMPS_ERR_ARG, "null handle");
  CMPS_TRY(use_device(h->impl->ctx));
  TuneStats s;
  CMPS_TRY(h->impl->autotune(&s));
  if (tuned) *tuned = s.tuned;
  if (cached) *cached = s.cached;
  if (ms_heuristic) *ms_heuristic = s.ms_heuristic;
  if (ms_best) *ms_best = s.ms_best;
  return CMPS_OK;
}

int cmps_heff_input_sectors(const cmps_heff* h, uint8_t* needed) {
  if (!h || !h->impl || !needed) return fail(CMPS_ERR_ARG, "null argument");
  const Heff& H = *h->impl;
  for (size_t m = 0; m < H.in_need.size(); ++m) needed[m] = H.in_need[m];
  return CMPS_OK;
}

int cmps_heff_set_windows(cmps_heff* h, const int64_t* in_base, int64_t in_len, const int64_t* out_base,
                          int64_t out_len) {
  if (!h || !h->impl || !in_base || !out_base) return fail(CMPS_ERR_ARG, "null argument");
  CMPS_TRY(use_device(h->impl->ctx));
  return h->impl->set_windows(in_base, in_len, out_base, out_len);
}

int cmps_heff_apply_theta_device(cmps_heff* h, const double* d_in, double* d_out, void* stream) {
  if (!h || !h->impl || !d_in || !d_out) return fail(CMPS_ERR_ARG, "null argument");
  if (d_in == d_out) return fail(CMPS_ERR_ARG, "theta-layout apply: in and out must be different arrays");
  Heff& H = *h->impl;
  CMPS_TRY(use_device(H.ctx));
  cudaStream_t st = stream ? (cudaStream_t)stream : H.ctx->stream;
  // views of the caller's arrays (planar: re plane, then im plane), in the
  // handle's windows (the theta layout unless cmps_heff_set_windows)
  Planar in, out;
  in.d = const_cast<double*>(d_in);
  in.len = H.in_len;
  out.d = d_out;
  out.len = H.out_len;
  int rc;
  if (is_split(H.precision)) {
    rc = apply_split_stage(H, 1, in, out, st);
    if (rc == CMPS_OK) rc = apply_split_stage(H, 2, in, out, st);
    if (rc == CMPS_OK) rc = H.add_projectors(in, out, st);
  } else {
    rc = H.apply_theta_fp64(in, out, st);
  }
  in.d = out.d = nullptr;
  return rc;
}

int cmps_heff_set_projectors(cmps_heff* h, int count, const double* tensors, const double* weights) {
  if (!h || !h->impl) return fail(CMPS_ERR_ARG, "null handle");
  CMPS_TRY(use_device(h->impl->ctx));
  return h->impl->set_projectors(count, tensors, weights);
}

int cmps_heff_theta_from_arpack(cmps_heff* h, const double* d_arpack, double* d_theta, void* stream) {
  if (!h || !h->impl || !d_arpack || !d_theta) return fail(CMPS_ERR_ARG, "null argument");
  Heff& H = *h->impl;
  CMPS_TRY(use_device(H.ctx));
  Planar out;
  out.d = d_theta;
  out.len = H.th.total;
  const int rc = H.pack(d_arpack, out, stream ? (cudaStream_t)stream : H.ctx->stream);
  out.d = nullptr;
  return rc;
}

int cmps_heff_theta_to_arpack(cmps_heff* h, const double* d_theta, double* d_arpack, void* stream) {
  if (!h || !h->impl || !d_arpack || !d_theta) return fail(CMPS_ERR_ARG, "null argument");
  Heff& H = *h->impl;
  CMPS_TRY(use_device(H.ctx));
  Planar in;
  in.d = const_cast<double*>(d_theta);
  in.len = H.th.total;
  const int rc = H.unpack(in, d_arpack, stream ? (cudaStream_t)stream : H.ctx->stream);
  in.d = nullptr;
  return rc;
}

int cmps_heff_time_stages(cmps_heff* h, const double* d_in, double* d_out, void* stream, int reps, double* ms) {
  if (!h || !h->impl || !d_in || !d_out || !ms || reps < 1) return fail(CMPS_ERR_ARG, "bad argument");
  Heff& H = *h->impl;
  CMPS_TRY(use_device(H.ctx));
  if (!H.whole()) return fail(CMPS_ERR_STATE, "stage timing: the matvec is sharded");
  cudaStream_t st = stream ? (cudaStream_t)stream : H.ctx->stream;
  cudaEvent_t ev[5];
  for (auto& e : ev) CMPS_CUDA(cudaEventCreate(&e));
  double acc[4] = {0, 0, 0, 0};
  int status = CMPS_OK;
  for (int r = 0; r < reps && status == CMPS_OK; ++r) {
    cudaEventRecord(ev[0], st);
    status = H.pack(d_in, H.x, st);
    cudaEventRecord(ev[1], st);
    if (status == CMPS_OK) status = H.apply_stage(1, H.x, H.y, st);
    cudaEventRecord(ev[2], st);
    if (status == CMPS_OK) status = H.apply_stage(2, H.x, H.y, st);
    cudaEventRecord(ev[3], st);
    if (status == CMPS_OK) status = H.unpack(H.y, d_out, st);
    cudaEventRecord(ev[4], st);
    if (cudaEventSynchronize(ev[4]) != cudaSuccess) status = fail(CMPS_ERR_CUDA, "stage timing failed");
    for (int k = 0; k < 4 && status == CMPS_OK; ++k) {
      float t = 0.f;
      cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
      acc[k] += t;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  for (int k = 0; k < 4; ++k) ms[k] = acc[k] / reps;
  if (status == CMPS_OK) status = split_error(H);
  return status;
}

int cmps_heff_status(cmps_heff* h) {
  if (!h || !h->impl) return fail(CMPS_ERR_ARG, "null handle");
  CMPS_TRY(use_device(h->impl->ctx));
  CMPS_CUDA(cudaStreamSynchronize(h->impl->ctx->stream));
  CMPS_CUDA(cudaDeviceSynchronize());
  return split_error(*h->impl);
}

int cmps_heff_flops(const cmps_heff* h, double* canonical, double* executed) {
  if (!h || !h->impl) return fail(CMPS_ERR_ARG, "null handle");
  const Heff& H = *h->impl;
  if (canonical) *canonical = H.flops_canonical;
  if (executed) {
    const bool canonical = H.precision == CMPS_FP64 ? H.order == CMPS_ORDER_CANONICAL : H.low_canonical;
    *executed = H.precision != CMPS_FP64 && H.ctc ? canonical_tc_flops(H)
                : canonical                        ? H.flops_canon
                                                   : H.flops_executed;
  }
  return CMPS_OK;
}

int cmps_heff_set_order(cmps_heff* h, int order) {
  if (!h || !h->impl) return fail(CMPS_ERR_ARG, "null handle");
  if (order != CMPS_ORDER_AUTO && order != CMPS_ORDER_FOLDED && order != CMPS_ORDER_CANONICAL)
    return fail(CMPS_ERR_ARG, "unknown contraction order");
  Heff& H = *h->impl;
  CMPS_TRY(use_device(H.ctx));
  CMPS_CUDA(cudaStreamSynchronize(H.ctx->stream));
  H.order_req = order;
  return H.select_order();
}

int cmps_heff_order(const cmps_heff* h, int* active, double* executed_folded, double* executed_canonical) {
  if (!h || !h->impl) return fail(CMPS_ERR_ARG, "null handle");
  const Heff& H = *h->impl;
  if (active) *active = H.order;
  if (executed_folded) *executed_folded = H.flops_folded;
  if (executed_canonical) *executed_canonical = H.flops_canon;
  return CMPS_OK;
}

int cmps_heff_split_form(const cmps_heff* h, int* form) {
  if (!h || !h->impl || !form) return fail(CMPS_ERR_ARG, "null argument");
  *form = split_form(*h->impl);
  return CMPS_OK;
}

int cmps_heff_set_precision(cmps_heff* h, int precision) {
  if (!h || !h->impl) return fail(CMPS_ERR_ARG, "null handle");
  if (precision != CMPS_FP64 && !is_split(precision)) return fail(CMPS_ERR_ARG, "unknown precision");
  CMPS_TRY(prepare_precision(h->impl.get(), precision));
  h->impl->precision = precision;
  return CMPS_OK;
}

int cmps_heff_eigs(cmps_heff* h, const double* guess, double tol, int max_restarts, int krylov_dim,
                   double* eval, double* evec, int* matvecs) {
  if (!h || !h->impl || !eval) return fail(CMPS_ERR_ARG, "null argument");
  if (!(tol > 0.0)) return fail(CMPS_ERR_ARG, "tolerance must be positive");
  CMPS_TRY(use_device(h->impl->ctx));
  return h->impl->eigs(guess, tol, max_restarts, krylov_dim, eval, evec, matvecs);
}

int cmps_heff_eigs_stats(const cmps_heff* h, int* split_matvecs, int* fp64_matvecs, int* cycles, double* ms3) {
  if (!h || !h->impl) return fail(CMPS_ERR_ARG, "null handle");
  const Heff::EigStats& s = h->impl->eig_stats;
  if (split_matvecs) *split_matvecs = s.mv_split;
  if (fp64_matvecs) *fp64_matvecs = s.mv_fp64;
  if (cycles) *cycles = s.cycles;
  if (ms3) {
    ms3[0] = s.ms_split;
    ms3[1] = s.ms_fp64;
    ms3[2] = s.ms_total;
  }
  return CMPS_OK;
}

int cmps_heff_set_theta(cmps_heff* h, const double* theta) {
  if (!h || !h->impl || !theta) return fail(CMPS_ERR_ARG, "null argument");
  Heff& H = *h->impl;
  CMPS_TRY(use_device(H.ctx));
  cudaStream_t st = H.ctx->stream;
  CMPS_CUDA(cudaMemcpyAsync(H.d_io, theta, sizeof(double) * 2 * H.n_allowed, cudaMemcpyHostToDevice, st));
  if (H.theta.len != H.th.total) CMPS_TRY(H.theta.alloc(H.th.total));
  CMPS_TRY(H.pack(H.d_io, H.theta, st));
  CMPS_CUDA(cudaStreamSynchronize(st));
  H.have_theta = true;
  return CMPS_OK;
}

}  // extern "C"
