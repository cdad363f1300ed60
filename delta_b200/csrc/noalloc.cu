// noalloc.cu -- delta_pairs_run_host_noalloc: the host-buffer pair-list entry point
// without any device allocation.
//
// Some callers cannot let a library call cudaMalloc: a host that hands all device memory
// to its own pooling allocator (a raw cudaMalloc there either fails for lack of memory or
// fragments the pool), and latency-bound loops that must not pay for an allocation or
// for the implicit device synchronisation that cudaMalloc/cudaFree can bring.  For them
// this entry point stages inputs and outputs in one fixed device array that is part of
// the library image: the CUDA driver reserves it (62.8 MiB) on each GPU when it loads the
// library's module there, and every GPU that loads the library holds it until the
// process exits.
//
// Host code may not use the array's name as a device address: on the host it names a
// stand-in object.  So the first call on a device, with that device current, looks the
// array's device address up with cudaGetSymbolAddress (which may also make the driver
// load the module there) and keeps it for that device.  That address stays valid for the
// life of the device's primary context; do not use this entry point across a
// cudaDeviceReset of the device.  Every call on a device shares the one array and the
// array keeps the previous call's contents: each call overwrites the entries it uses
// before reading them, so nothing has to start at zero, but calls that overlap on the GPU
// (other streams, other threads, other contexts on the same device) race for the array.
#include <mutex>

#include "internal.h"

namespace delta {

// 25 doubles (a: 9, b: 9, p: 3, q: 3, dist: 1) and one flag byte per pair.
constexpr int64_t kNoAllocMaxPairs = DELTA_NOALLOC_MAX_PAIRS;
constexpr size_t kNoAllocBytes = (size_t)kNoAllocMaxPairs * (25 * sizeof(double) + 1);

static __device__ __align__(256) unsigned char g_noalloc_staging[kNoAllocBytes];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
void *g_noalloc_ptr[kMaxDevices] = {};
}  // namespace

// Device address of the staging array on `device` (which must be current).
static delta_status noalloc_staging(int device, void **out) {
  if (device < 0 || device >= kMaxDevices) return set_error(DELTA_ERR_INVALID, "noalloc: device ordinal too large");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_staging);
    if (e != cudaSuccess) return cuda_error(e, "noalloc: cudaGetSymbolAddress");
    g_noalloc_ptr[device] = p;
  }
  *out = g_noalloc_ptr[device];
  return DELTA_OK;
}

}  // namespace delta

using namespace delta;

extern "C" delta_status delta_pairs_run_host_noalloc(delta_ctx *ctx, int method, int precision, int64_t n,
                                                     const double *a, const double *b, int64_t ld, double max_error,
                                                     double *p, double *q, double *dist, uint8_t *flags) {
  if (!ctx) return set_error(DELTA_ERR_INVALID, "null context");
  if (method < DELTA_BF || method > DELTA_BF_CERT) return set_error(DELTA_ERR_INVALID, "unknown method");
  if (precision != DELTA_F64 && precision != DELTA_F32) return set_error(DELTA_ERR_INVALID, "unknown precision");
  if (n < 0 || ld < n) return set_error(DELTA_ERR_INVALID, "need 0 <= n <= ld");
  if (n > kNoAllocMaxPairs)
    return set_error(DELTA_ERR_CAPACITY, "delta_pairs_run_host_noalloc: n exceeds DELTA_NOALLOC_MAX_PAIRS (" +
                                             std::to_string(kNoAllocMaxPairs) + ")");
  if (n == 0) return DELTA_OK;
  if (!a || !b || !p || !q || !dist) return set_error(DELTA_ERR_INVALID, "null buffer");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
  void *base = nullptr;
  delta_status st = noalloc_staging(ctx->device, &base);
  if (st != DELTA_OK) return st;
  // layout for this call: a(9n) b(9n) p(3n) q(3n) dist(n) flags(n)
  const size_t nd = (size_t)n;
  double *da = (double *)base, *db = da + 9 * nd, *dp = db + 9 * nd, *dq = dp + 3 * nd, *dd = dq + 3 * nd;
  uint8_t *df = (uint8_t *)(dd + nd);
  cudaStream_t s = ctx->stream;
  e = cudaMemcpy2DAsync(da, sizeof(double) * nd, a, sizeof(double) * ld, sizeof(double) * nd, 9,
                        cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(db, sizeof(double) * nd, b, sizeof(double) * ld, sizeof(double) * nd, 9,
                          cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return cuda_error(e, "noalloc H2D");
  e = launch_pairs_cfg(method, precision, s, n, da, db, n, max_error, dp, dq, dd, flags ? df : nullptr,
                       ctx_pair_launch(ctx, method, precision));
  if (e != cudaSuccess) return cuda_error(e, "noalloc pairs kernel launch");
  ctx->launches += 1;
  e = cudaMemcpy2DAsync(p, sizeof(double) * ld, dp, sizeof(double) * nd, sizeof(double) * nd, 3,
                        cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(q, sizeof(double) * ld, dq, sizeof(double) * nd, sizeof(double) * nd, 3,
                          cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dist, dd, sizeof(double) * nd, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && flags) e = cudaMemcpyAsync(flags, df, nd, cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return cuda_error(e, "noalloc D2H");
  return cuda_error(cudaStreamSynchronize(s), "noalloc sync");
}
