// capi.cu -- context management and the pair-list entry points of the C ABI.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <algorithm>

#include "internal.h"

namespace delta {

static thread_local std::string g_last_error;

delta_status set_error(delta_status st, const std::string &msg) {
  g_last_error = msg;
  return st;
}

delta_status cuda_error(cudaError_t e, const char *where) {
  if (e == cudaSuccess) return DELTA_OK;
  return set_error(e == cudaErrorMemoryAllocation ? DELTA_ERR_NOMEM : DELTA_ERR_CUDA,
                   std::string(where) + ": " + cudaGetErrorString(e));
}

delta_status ctx_scratch(delta_ctx *ctx, int slot, size_t bytes, void **out) {
  delta_buffer &b = ctx->scratch[slot];
  if (b.bytes < bytes) {
    if (b.ptr) {
      cudaError_t e = cudaStreamSynchronize(ctx->stream);
      if (e != cudaSuccess) return cuda_error(e, "scratch sync");
      cudaFree(b.ptr);
      b.ptr = nullptr;
      b.bytes = 0;
    }
    size_t want = bytes + bytes / 4 + 256;
    cudaError_t e = cudaMalloc(&b.ptr, want);
    if (e != cudaSuccess) return cuda_error(e, "scratch cudaMalloc");
    b.bytes = want;
  }
  *out = b.ptr;
  return DELTA_OK;
}

delta_status host_pipeline(
    delta_ctx *ctx, int64_t n, const double *a, const double *b, int64_t ld, double *p, double *q, double *dist,
    uint8_t *flags,
    const std::function<delta_status(int64_t, int64_t, const double *, const double *, int64_t, double *, double *,
                                     double *, uint8_t *)> &run,
    const std::function<delta_status(int)> &after) {
  // device layout: a(9n) b(9n) p(3n) q(3n) dist(n) | flags(n)
  const size_t nd = (size_t)n;
  void *buf = nullptr, *fbuf = nullptr;
  delta_status st;
  if ((st = ctx_scratch(ctx, 0, sizeof(double) * 25 * nd, &buf)) != DELTA_OK) return st;
  if ((st = ctx_scratch(ctx, 1, nd, &fbuf)) != DELTA_OK) return st;
  double *da = (double *)buf, *db = da + 9 * nd, *dp = db + 9 * nd, *dq = dp + 3 * nd, *dd = dq + 3 * nd;
  uint8_t *df = (uint8_t *)fbuf;
  cudaError_t e = cudaSuccess;
  if (!ctx->copy_in && (e = cudaStreamCreateWithFlags(&ctx->copy_in, cudaStreamNonBlocking)) != cudaSuccess)
    return cuda_error(e, "copy stream");
  if (!ctx->copy_out && (e = cudaStreamCreateWithFlags(&ctx->copy_out, cudaStreamNonBlocking)) != cudaSuccess)
    return cuda_error(e, "copy stream");
  for (auto &ev : ctx->events)
    if (!ev && (e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess)
      return cuda_error(e, "copy events");
  // up to 15 chunks of at least 2^18 pairs (the first H2D and the last D2H are not
  // overlapped, so more chunks leave less of them exposed); event 0 starts the H2D after
  // the context's earlier work, 1+3k and 2+3k mark the end of chunk k's H2D and compute,
  // the last one the end of the copies
  const int64_t min_chunk = 1 << 18;
  int chunks = (int)std::min<int64_t>(15, std::max<int64_t>(1, n / min_chunk));
  const int64_t chunk = (n + chunks - 1) / chunks;
  chunks = (int)((n + chunk - 1) / chunk);
  cudaEvent_t *ev = ctx->events;
  if ((e = cudaEventRecord(ev[0], ctx->stream)) != cudaSuccess ||
      (e = cudaStreamWaitEvent(ctx->copy_in, ev[0], 0)) != cudaSuccess)
    return cuda_error(e, "pipeline start");
  const size_t hp = sizeof(double) * (size_t)ld, dp_pitch = sizeof(double) * nd;
  for (int k = 0; k < chunks; ++k) {
    const int64_t c0 = k * chunk, nc = std::min<int64_t>(chunk, n - c0);
    const size_t w = sizeof(double) * (size_t)nc;
    e = cudaMemcpy2DAsync(da + c0, dp_pitch, a + c0, hp, w, 9, cudaMemcpyHostToDevice, ctx->copy_in);
    if (e == cudaSuccess) e = cudaMemcpy2DAsync(db + c0, dp_pitch, b + c0, hp, w, 9, cudaMemcpyHostToDevice, ctx->copy_in);
    if (e == cudaSuccess) e = cudaEventRecord(ev[1 + 3 * k], ctx->copy_in);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->stream, ev[1 + 3 * k], 0);
    if (e != cudaSuccess) return cuda_error(e, "pipeline H2D");
    if ((st = run(c0, nc, da + c0, db + c0, (int64_t)nd, dp + c0, dq + c0, dd + c0, flags ? df + c0 : nullptr)) !=
        DELTA_OK)
      return st;
    if (after && (st = after(k)) != DELTA_OK) return st;
    e = cudaEventRecord(ev[2 + 3 * k], ctx->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->copy_out, ev[2 + 3 * k], 0);
    if (e == cudaSuccess)
      e = cudaMemcpy2DAsync(p + c0, hp, dp + c0, dp_pitch, w, 3, cudaMemcpyDeviceToHost, ctx->copy_out);
    if (e == cudaSuccess)
      e = cudaMemcpy2DAsync(q + c0, hp, dq + c0, dp_pitch, w, 3, cudaMemcpyDeviceToHost, ctx->copy_out);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dist + c0, dd + c0, w, cudaMemcpyDeviceToHost, ctx->copy_out);
    if (e == cudaSuccess && flags)
      e = cudaMemcpyAsync(flags + c0, df + c0, (size_t)nc, cudaMemcpyDeviceToHost, ctx->copy_out);
    if (e != cudaSuccess) return cuda_error(e, "pipeline D2H");
  }
  // the context stream continues after the last copy
  cudaEvent_t last = ev[sizeof(ctx->events) / sizeof(ctx->events[0]) - 1];
  if ((e = cudaEventRecord(last, ctx->copy_out)) != cudaSuccess ||
      (e = cudaStreamWaitEvent(ctx->stream, last, 0)) != cudaSuccess)
    return cuda_error(e, "pipeline end");
  return cuda_error(cudaStreamSynchronize(ctx->stream), "pipeline sync");
}

delta_status ctx_pinned(delta_ctx *ctx, size_t bytes, void **out) {
  if (ctx->pinned_bytes < bytes) {
    if (ctx->pinned) {
      cudaError_t e = cudaStreamSynchronize(ctx->stream);
      if (e != cudaSuccess) return cuda_error(e, "pinned sync");
      cudaFreeHost(ctx->pinned);
      ctx->pinned = nullptr;
      ctx->pinned_bytes = 0;
    }
    cudaError_t e = cudaMallocHost(&ctx->pinned, bytes);
    if (e != cudaSuccess) return cuda_error(e, "cudaMallocHost");
    ctx->pinned_bytes = bytes;
  }
  *out = ctx->pinned;
  return DELTA_OK;
}

}  // namespace delta

using namespace delta;

extern "C" {

const char *delta_last_error(void) { return g_last_error.c_str(); }
const char *delta_version(void) { return "delta_b200 0.1 (sm_100a)"; }

delta_status delta_create(delta_ctx **out, int device, void *stream) {
  if (!out) return set_error(DELTA_ERR_INVALID, "delta_create: null output");
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) return cuda_error(e, "cudaGetDeviceCount");
  if (device < 0 || device >= n) return set_error(DELTA_ERR_INVALID, "delta_create: bad device");
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
  delta_ctx *c = new delta_ctx();
  c->device = device;
  c->stream = (cudaStream_t)stream;
  *out = c;
  return DELTA_OK;
}

delta_status delta_destroy(delta_ctx *ctx) {
  if (!ctx) return DELTA_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (auto &b : ctx->scratch)
    if (b.ptr) cudaFree(b.ptr);
  for (auto &ev : ctx->events)
    if (ev) cudaEventDestroy(ev);
  if (ctx->copy_in) cudaStreamDestroy(ctx->copy_in);
  if (ctx->copy_out) cudaStreamDestroy(ctx->copy_out);
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  if (ctx->gemm_err) cudaFree(ctx->gemm_err);
  delete ctx;
  return DELTA_OK;
}

delta_status delta_set_stream(delta_ctx *ctx, void *stream) {
  if (!ctx) return set_error(DELTA_ERR_INVALID, "null context");
  ctx->stream = (cudaStream_t)stream;
  return DELTA_OK;
}

delta_status delta_synchronize(delta_ctx *ctx) {
  if (!ctx) return set_error(DELTA_ERR_INVALID, "null context");
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess || !ctx->gemm_err) return cuda_error(e, "cudaStreamSynchronize");
  // a tcgen05 GEMM whose bounded wait gave up (its output was set to NaN) since the last check
  int flag = 0;
  if ((e = cudaMemcpy(&flag, ctx->gemm_err, sizeof(int), cudaMemcpyDeviceToHost)) != cudaSuccess)
    return cuda_error(e, "gemm flag");
  if (!flag) return DELTA_OK;
  cudaMemset(ctx->gemm_err, 0, sizeof(int));
  return set_error(DELTA_ERR_TIMEOUT, "tcgen05 GEMM: bounded wait for the tensor cores gave up");
}

int64_t delta_launch_count(const delta_ctx *ctx) { return ctx ? ctx->launches : 0; }

static delta_status check_pairs(delta_ctx *ctx, int method, int precision, int64_t n, const void *a, const void *b,
                                int64_t ld, const void *p, const void *q, const void *dist) {
  if (!ctx) return set_error(DELTA_ERR_INVALID, "null context");
  if (method < DELTA_BF || method > DELTA_BF_CERT) return set_error(DELTA_ERR_INVALID, "unknown method");
  if (precision != DELTA_F64 && precision != DELTA_F32) return set_error(DELTA_ERR_INVALID, "unknown precision");
  if (n < 0 || ld < n) return set_error(DELTA_ERR_INVALID, "need 0 <= n <= ld");
  if (n > 0 && (!a || !b || !p || !q || !dist)) return set_error(DELTA_ERR_INVALID, "null buffer");
  return DELTA_OK;
}

delta_status delta_pairs_run(delta_ctx *ctx, int method, int precision, int64_t n, const double *a,
                             const double *b, int64_t ld, double max_error, double *p, double *q, double *dist,
                             uint8_t *flags) {
  delta_status st = check_pairs(ctx, method, precision, n, a, b, ld, p, q, dist);
  if (st != DELTA_OK || n == 0) return st;
  cudaError_t e = launch_pairs_cfg(method, precision, ctx->stream, n, a, b, ld, max_error, p, q, dist, flags,
                                   ctx_pair_launch(ctx, method, precision));
  if (e != cudaSuccess) return cuda_error(e, "pairs kernel launch");
  ctx->launches += 1;
  return DELTA_OK;
}

delta_status delta_set_pair_launch(delta_ctx *ctx, int method, int precision, int32_t threads,
                                   int32_t blocks_per_sm) {
  if (!ctx || method < DELTA_BF || method > DELTA_BF_CERT || (precision != 0 && precision != 1))
    return set_error(DELTA_ERR_INVALID, "delta_set_pair_launch: bad method/precision");
  if (!(threads == 64 || threads == 128 || threads == 256) || blocks_per_sm < 0 ||
      threads > pair_max_threads(method, precision))
    return set_error(DELTA_ERR_INVALID, "delta_set_pair_launch: unsupported launch shape");
  ctx->pair_launch[method][precision] = PairLaunch{threads, blocks_per_sm};
  ctx->pair_launch_set[method][precision] = true;
  return DELTA_OK;
}

delta_status delta_set_cull_launch(delta_ctx *ctx, int32_t cull_blocks_per_sm, int32_t survivor_blocks_per_sm) {
  if (!ctx || cull_blocks_per_sm < 0 || survivor_blocks_per_sm < 0)
    return set_error(DELTA_ERR_INVALID, "delta_set_cull_launch: bad argument");
  ctx->cull_blocks_per_sm = cull_blocks_per_sm;
  ctx->surv_blocks_per_sm = survivor_blocks_per_sm;
  ctx->launch_epoch += 1;
  return DELTA_OK;
}

delta_status delta_autotune_pairs(delta_ctx *ctx, int method, int precision, int64_t n, const double *a,
                                  const double *b, int64_t ld, double max_error, double *p, double *q, double *dist,
                                  uint8_t *flags, int32_t *threads_out, int32_t *blocks_per_sm_out, float *ms_out) {
  delta_status st = check_pairs(ctx, method, precision, n, a, b, ld, p, q, dist);
  if (st != DELTA_OK) return st;
  if (n == 0) return set_error(DELTA_ERR_INVALID, "delta_autotune_pairs: empty sample");
  std::vector<PairLaunch> cand;
  if (method == DELTA_BF_CERT) {
    for (int t : {64, 128})
      for (int b : {2, 4, 8, 16}) cand.push_back(PairLaunch{t, b});
  } else {
    for (int t : {64, 128, 256})
      for (int b : {4, 8, 16, 32, 0})  // 0: one thread per pair
        if (t <= pair_max_threads(method, precision)) cand.push_back(PairLaunch{t, b});
  }
  cudaEvent_t e0, e1;
  cudaError_t e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  if (e != cudaSuccess) return cuda_error(e, "autotune events");
  float best = 1e30f;
  PairLaunch bestc = default_pair_launch(method);
  for (const PairLaunch &c : cand) {
    e = launch_pairs_cfg(method, precision, ctx->stream, n, a, b, ld, max_error, p, q, dist, flags, c);  // warm-up
    if (e == cudaSuccess) e = cudaEventRecord(e0, ctx->stream);
    for (int k = 0; k < 3 && e == cudaSuccess; ++k)
      e = launch_pairs_cfg(method, precision, ctx->stream, n, a, b, ld, max_error, p, q, dist, flags, c);
    if (e == cudaSuccess) e = cudaEventRecord(e1, ctx->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e != cudaSuccess) break;
    ctx->launches += 4;
    if (ms / 3 < best) {
      best = ms / 3;
      bestc = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return cuda_error(e, "autotune");
  ctx->pair_launch[method][precision] = bestc;
  ctx->pair_launch_set[method][precision] = true;
  if (threads_out) *threads_out = bestc.threads;
  if (blocks_per_sm_out) *blocks_per_sm_out = bestc.blocks_per_sm;
  if (ms_out) *ms_out = best;
  return DELTA_OK;
}

delta_status delta_pairs_run_host(delta_ctx *ctx, int method, int precision, int64_t n, const double *a,
                                  const double *b, int64_t ld, double max_error, double *p, double *q, double *dist,
                                  uint8_t *flags) {
  delta_status st = check_pairs(ctx, method, precision, n, a, b, ld, p, q, dist);
  if (st != DELTA_OK || n == 0) return st;
  const PairLaunch cfg = ctx_pair_launch(ctx, method, precision);
  return host_pipeline(ctx, n, a, b, ld, p, q, dist, flags,
                       [&](int64_t, int64_t nc, const double *da, const double *db, int64_t ldd, double *dp,
                           double *dq, double *dd, uint8_t *df) -> delta_status {
                         cudaError_t e = launch_pairs_cfg(method, precision, ctx->stream, nc, da, db, ldd, max_error,
                                                          dp, dq, dd, df, cfg);
                         ctx->launches += 1;
                         return cuda_error(e, "pairs kernel launch");
                       });
}

delta_status delta_detect(delta_ctx *ctx, int driver, int precision, const delta_meshes *meshes,
                          const int32_t *pair_a, const int32_t *pair_b, int64_t n_pairs,
                          const delta_contacts *out, int64_t *n_out, delta_stats *stats) {
  if (!ctx || !meshes || !out || !n_out) return set_error(DELTA_ERR_INVALID, "delta_detect: null argument");
  if (driver < DELTA_DRV_BF || driver > DELTA_DRV_LEARNED) return set_error(DELTA_ERR_INVALID, "unknown driver");
  if (precision != DELTA_F64 && precision != DELTA_F32) return set_error(DELTA_ERR_INVALID, "unknown precision");
  if (n_pairs < 0 || out->capacity < 0) return set_error(DELTA_ERR_INVALID, "negative size");
  *n_out = 0;
  if (stats) std::memset(stats, 0, sizeof(*stats));
  if (n_pairs == 0) return DELTA_OK;
  if (!pair_a || !pair_b || !meshes->tri_offset || !meshes->x || !meshes->y || !meshes->z || !meshes->eps ||
      !meshes->friction || !meshes->id || meshes->n_bodies <= 0)
    return set_error(DELTA_ERR_INVALID, "delta_detect: incomplete meshes or pairs");
  if (out->capacity > 0 && (!out->x || !out->normal || !out->P || !out->Q || !out->depth || !out->eps_total ||
                            !out->master || !out->slave || !out->tri_a || !out->tri_b || !out->penetration ||
                            !out->friction))
    return set_error(DELTA_ERR_INVALID, "delta_detect: incomplete contact buffer");
  return detect_run(ctx, driver, precision, *meshes, pair_a, pair_b, n_pairs, out, n_out, stats, nullptr);
}

}  // extern "C"
