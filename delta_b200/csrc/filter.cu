// filter.cu -- contact de-duplication (delta/contact/filter.cpp) on the GPU.
//
// filterNewContacts (filter.cpp:80-101) keeps a contact unless an earlier kept contact of
// the same particle pair lies within eps on every coordinate; the rule is sequential (a
// dropped contact drops nothing), so each particle pair's run of contacts is one warp's
// work: contacts in order, the warp's lanes testing the earlier survivors 32 at a time.
// filterOldContacts (filter.cpp:3-78) drops a new contact near any stored contact of the
// same pair: one thread per new contact, the stored contacts of its pair found by binary
// search over their sorted (master, slave) keys.  The comparisons are the reference's
// (|a - b| < eps on each coordinate, FP64), so the flags equal its results exactly.
#include <cub/cub.cuh>

#include "internal.h"

namespace delta {
namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ bool near3(const double *x, int64_t ld, int64_t i, const double *y, int64_t ldy,
                                      int64_t j, double eps) {
  return fabs(x[i] - y[j]) < eps && fabs(x[ld + i] - y[ldy + j]) < eps && fabs(x[2 * ld + i] - y[2 * ldy + j]) < eps;
}

__device__ __forceinline__ uint64_t pair_key(int32_t m, int32_t s) {
  return ((uint64_t)(uint32_t)m << 32) | (uint64_t)(uint32_t)s;
}

// 1 where a run of equal (master, slave) starts
__global__ void k_run_heads(int64_t n, const int32_t *__restrict__ m, const int32_t *__restrict__ s,
                            uint8_t *__restrict__ head) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) head[i] = (i == 0 || m[i] != m[i - 1] || s[i] != s[i - 1]) ? 1 : 0;
}

// one warp per run: contacts in order, each tested against the run's earlier survivors
__global__ void k_filter_new(int64_t n, const double *__restrict__ x, int64_t ld, const int64_t *__restrict__ start,
                             const int64_t *__restrict__ n_runs, double eps, uint8_t *keep) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t runs = *n_runs;
  for (int64_t r = warp; r < runs; r += nwarps) {
    const int64_t s = start[r], e = r + 1 < runs ? start[r + 1] : n;
    for (int64_t i = s; i < e; ++i) {
      bool hit = false;
      for (int64_t j = s + lane; j < i && !hit; j += 32) hit = keep[j] && near3(x, ld, i, x, ld, j, eps);
      hit = __any_sync(kFull, hit);
      if (lane == 0) keep[i] = hit ? 0 : 1;
      __syncwarp();
    }
  }
}

__global__ void k_pair_keys(int64_t n, const int32_t *__restrict__ m, const int32_t *__restrict__ s,
                            uint64_t *__restrict__ key, int64_t *__restrict__ idx) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    key[i] = pair_key(m[i], s[i]);
    idx[i] = i;
  }
}

__global__ void k_filter_old(int64_t ns, const double *__restrict__ xs, int64_t lds, const uint64_t *__restrict__ skey,
                             const int64_t *__restrict__ sidx, int64_t nn, const double *__restrict__ xn,
                             int64_t ldn, const int32_t *__restrict__ mn, const int32_t *__restrict__ sn, double eps,
                             uint8_t *__restrict__ keep) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  const uint64_t k = pair_key(mn[i], sn[i]);
  int64_t lo = 0, hi = ns;  // first stored key >= k
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (skey[mid] < k) lo = mid + 1;
    else hi = mid;
  }
  bool hit = false;
  for (int64_t j = lo; j < ns && skey[j] == k && !hit; ++j) hit = near3(xn, ldn, i, xs, lds, sidx[j], eps);
  keep[i] = hit ? 0 : 1;
}

inline unsigned blocks_for(int64_t n, int t = 256) { return (unsigned)std::max<int64_t>(1, (n + t - 1) / t); }

bool contacts_ok(const delta_contacts *c, int64_t n) {
  return c && n >= 0 && n <= c->capacity && (n == 0 || (c->x && c->master && c->slave));
}

}  // namespace
}  // namespace delta

using namespace delta;

extern "C" {

delta_status delta_filter_new_contacts(delta_ctx *ctx, const delta_contacts *c, int64_t n, double eps,
                                       uint8_t *keep) {
  if (!ctx || !contacts_ok(c, n) || (n > 0 && !keep) || !(eps >= 0.0))
    return set_error(DELTA_ERR_INVALID, "delta_filter_new_contacts: bad argument");
  if (n == 0) return DELTA_OK;
  // scratch: run heads (n bytes) | run starts (8n) | run count (8) | cub temp
  size_t tb = 0;
  cub::CountingInputIterator<int64_t> it(0);
  cudaError_t e = cub::DeviceSelect::Flagged(nullptr, tb, it, (const uint8_t *)nullptr, (int64_t *)nullptr,
                                             (int64_t *)nullptr, n, ctx->stream);
  if (e != cudaSuccess) return cuda_error(e, "filter: temp size");
  const size_t off_start = ((size_t)n + 255) / 256 * 256, off_count = off_start + 8 * (size_t)n,
               off_temp = off_count + 256;
  void *buf;
  delta_status st = ctx_scratch(ctx, 17, off_temp + tb, &buf);
  if (st != DELTA_OK) return st;
  char *base = static_cast<char *>(buf);
  uint8_t *head = reinterpret_cast<uint8_t *>(base);
  int64_t *start = reinterpret_cast<int64_t *>(base + off_start);
  int64_t *runs = reinterpret_cast<int64_t *>(base + off_count);
  k_run_heads<<<blocks_for(n), 256, 0, ctx->stream>>>(n, c->master, c->slave, head);
  if ((e = cub::DeviceSelect::Flagged(base + off_temp, tb, it, head, start, runs, n, ctx->stream)) != cudaSuccess)
    return cuda_error(e, "filter: runs");
  // one warp per run; at most n runs, grid capped at 32 warps per SM
  const int64_t warps = std::min<int64_t>(n, (int64_t)kNumSMs * 32);
  k_filter_new<<<blocks_for(warps * 32, 128), 128, 0, ctx->stream>>>(n, c->x, c->capacity, start, runs, eps, keep);
  ctx->launches += 2;
  return cuda_error(cudaGetLastError(), "delta_filter_new_contacts");
}

delta_status delta_filter_old_contacts(delta_ctx *ctx, const delta_contacts *stored, int64_t n_stored,
                                       const delta_contacts *fresh, int64_t n_fresh, double eps, uint8_t *keep) {
  if (!ctx || !contacts_ok(stored, n_stored) || !contacts_ok(fresh, n_fresh) || (n_fresh > 0 && !keep) ||
      !(eps >= 0.0))
    return set_error(DELTA_ERR_INVALID, "delta_filter_old_contacts: bad argument");
  if (n_fresh == 0) return DELTA_OK;
  // scratch: keys (8 ns) | sorted keys (8 ns) | idx (8 ns) | sorted idx (8 ns) | cub temp
  const int64_t ns = n_stored;
  size_t tb = 0;
  cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, tb, (const uint64_t *)nullptr, (uint64_t *)nullptr,
                                                  (const int64_t *)nullptr, (int64_t *)nullptr, std::max<int64_t>(ns, 1),
                                                  0, 64, ctx->stream);
  if (e != cudaSuccess) return cuda_error(e, "filter: sort size");
  const size_t seg = ((size_t)std::max<int64_t>(ns, 1) * 8 + 255) / 256 * 256;
  void *buf;
  delta_status st = ctx_scratch(ctx, 18, 4 * seg + tb, &buf);
  if (st != DELTA_OK) return st;
  char *base = static_cast<char *>(buf);
  uint64_t *key = reinterpret_cast<uint64_t *>(base), *skey = reinterpret_cast<uint64_t *>(base + seg);
  int64_t *idx = reinterpret_cast<int64_t *>(base + 2 * seg), *sidx = reinterpret_cast<int64_t *>(base + 3 * seg);
  if (ns > 0) {
    k_pair_keys<<<blocks_for(ns), 256, 0, ctx->stream>>>(ns, stored->master, stored->slave, key, idx);
    if ((e = cub::DeviceRadixSort::SortPairs(base + 4 * seg, tb, key, skey, idx, sidx, ns, 0, 64, ctx->stream)) !=
        cudaSuccess)
      return cuda_error(e, "filter: sort");
    ctx->launches += 1;
  }
  k_filter_old<<<blocks_for(n_fresh), 256, 0, ctx->stream>>>(ns, ns > 0 ? stored->x : nullptr, stored->capacity, skey,
                                                             sidx, n_fresh, fresh->x, fresh->capacity, fresh->master,
                                                             fresh->slave, eps, keep);
  ctx->launches += 1;
  return cuda_error(cudaGetLastError(), "delta_filter_old_contacts");
}

}  // extern "C"
