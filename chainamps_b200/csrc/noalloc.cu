// H_eff matvec that allocates nothing: the variant of cmps_heff_apply_device
// for callers that cannot call cudaMalloc at call time.
//
// The matvec needs scratch beyond its input and output: the wavefunction in
// sector-block form (gathered input and stage-2 output) and the stage-1
// intermediate T.  cmps_heff_apply_device keeps that scratch in the handle.
// This variant takes it from one file-scope device array instead, of a fixed
// maximum size, so the call itself never allocates, frees or calls an
// allocating library routine.
//
// Who needs it: an eigensolver callback (ARPACK's reverse-communication MV,
// called hundreds of times per DMRG step) running inside a host application
// whose device memory is handed out by its own pool or caching allocator
// (a PyTorch process, an MPI code that reserves HBM up front), where a
// cudaMalloc from inside the callback would fail once the pool owns the
// memory, or would add an allocation plus a device-wide synchronisation to
// every Arnoldi iteration.
#include <cuda_runtime.h>

#include <mutex>

#include "heff.h"

namespace cmps {

// Maximum scratch of the no-allocation matvec: 4 Mi doubles (32 MiB).  It is
// a static device array, so every GPU that loads this library reserves it
// until the process exits.  Layout per call, in doubles: gathered input
// (2 * n), stage-1 intermediate (2 * t), stage-2 output (2 * n), where n is
// the number of allowed wavefunction entries and t the size of T.
constexpr int64_t kNoAllocScratchDoubles = 4ll * 1024 * 1024;
static __device__ __align__(256) double g_matvec_scratch[kNoAllocScratchDoubles];

// In host code g_matvec_scratch is only a host-side stand-in for the symbol;
// the device address comes from cudaGetSymbolAddress, once per device, with
// that device current.
static std::mutex g_scratch_mu;
static double* g_scratch_ptr[64] = {nullptr};

static int scratch_address(int device, double** out) {
  if (device < 0 || device >= 64) return fail(CMPS_ERR_ARG, "device ordinal out of range for the static scratch");
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_matvec_scratch);
    if (e != cudaSuccess || !p)
      return fail(CMPS_ERR_CUDA, std::string("cudaGetSymbolAddress(static matvec scratch): ") + cudaGetErrorString(e));
    g_scratch_ptr[device] = (double*)p;
  }
  *out = g_scratch_ptr[device];
  return CMPS_OK;
}

}  // namespace cmps

using namespace cmps;

extern "C" int cmps_heff_apply_device_noalloc(cmps_heff* h, const double* d_in, double* d_out, void* stream) {
  if (!h || !h->impl || !d_in || !d_out) return fail(CMPS_ERR_ARG, "null argument");
  Heff& H = *h->impl;
  if (H.precision != CMPS_FP64)
    return fail(CMPS_ERR_ARG, "the no-allocation matvec runs the FP64 path only; set CMPS_FP64 on the handle");
  if (H.proj_np || !H.whole())
    return fail(CMPS_ERR_ARG, "the no-allocation matvec runs the plain unsharded operator (no projectors)");
  const int64_t need = 4 * H.th.total + 2 * H.t_len;
  if (need > kNoAllocScratchDoubles)
    return fail(CMPS_ERR_ARG, "no-allocation matvec: this H_eff needs " + std::to_string(need * 8) +
                                  " bytes of scratch, above the static maximum of " +
                                  std::to_string(kNoAllocScratchDoubles * 8) + " bytes");
  CMPS_CUDA(cudaSetDevice(H.device));
  cudaGetLastError();  // drop a stale non-sticky error of an unrelated earlier call
  double* base = nullptr;
  CMPS_TRY(scratch_address(H.device, &base));
  cudaStream_t st = stream ? (cudaStream_t)stream : H.ctx->stream;
  // non-owning views into the static array
  Planar x, t, y;
  x.d = base;
  x.len = H.th.total;
  t.d = base + 2 * H.th.total;
  t.len = H.t_len;
  y.d = t.d + 2 * H.t_len;
  y.len = H.th.total;
  CMPS_TRY(H.pack(d_in, x, st));
  CMPS_TRY(launch_zgemm_fp64(H.stage1, false, false, H.LP, x, t, st));
  CMPS_TRY(launch_zgemm_fp64(H.stage2, false, false, t, H.RP, y, st));
  CMPS_TRY(H.unpack(y, d_out, st));
  return CMPS_OK;
}
