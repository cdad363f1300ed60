// internal.h -- declarations shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <string>

#include "delta_b200.h"

namespace delta {

constexpr int kNumSMs = 148;  // B200

// Launch shape of a pair-list kernel: threads per block (64, 128, 256) and the grid
// cap in blocks per SM (cert: in units of the occupancy limit).
// Launch shape of a pair kernel: threads per block and the grid cap in blocks per SM
// (0: no cap, one thread per pair).
struct PairLaunch {
  int threads = 256;
  int blocks_per_sm = 32;
};
inline PairLaunch default_pair_launch(int method) {
  PairLaunch c;
  if (method == 5) {
    c.threads = 128;
    c.blocks_per_sm = 8;
  } else if (method == 0) {
    c.threads = 128;
    c.blocks_per_sm = 0;
  }
  return c;
}
// The largest threads per block the pair kernel of (method, precision) takes (pairs.cu).
int pair_max_threads(int method, int precision);
// Position of coordinate c (0..17: a's 9, then b's 9) of list entry j in the exact
// solver's staging buffer: tiles of 32 entries, each tile 18 rows of 32 doubles, so one
// warp's 32 consecutive entries read one contiguous 4.6 KB tile (rather than 18 planes a
// power-of-two stride apart). A buffer for m entries holds kStageCoords * round_up(m, 32).
constexpr int kStageCoords = 18;
__host__ __device__ __forceinline__ int64_t stage_at(int64_t j, int c) {
  return ((j >> 5) * kStageCoords + c) * 32 + (j & 31);
}
inline size_t stage_doubles(int64_t m) { return (size_t)kStageCoords * (size_t)((m + 31) & ~(int64_t)31); }
// DELTA_BF_CERT over pairs idx[0 .. *count) (count read on the device, at most max_count);
// with `stage`, the coordinates of entry j come from stage[stage_at(j, c)].
cudaError_t launch_cert_indexed(cudaStream_t s, const uint32_t *count, int64_t max_count, const uint32_t *idx,
                                const double *a, const double *b, int64_t ld, double *p, double *q, double *dist,
                                PairLaunch cfg, const double *stage = nullptr);
cudaError_t launch_pairs_cfg(int method, int precision, cudaStream_t s, int64_t n, const double *a, const double *b,
                             int64_t ld, double max_error, double *p, double *q, double *dist, uint8_t *flags,
                             PairLaunch cfg);

// Pair-list launcher (pairs.cu), default launch shape.
cudaError_t launch_pairs(int method, int precision, cudaStream_t s, int64_t n, const double *a, const double *b,
                         int64_t ld, double max_error, double *p, double *q, double *dist, uint8_t *flags);

struct Pose;  // pose.cuh

// Particle-pair drivers (detect.cu).  `pose`: for the certified driver, the bodies' poses
// from which the current vertices and the body boxes are formed (the meshes' vertex arrays
// need not be current), or null (then the meshes' vertices are read and the body boxes
// computed from them).
delta_status detect_run(delta_ctx *ctx, int driver, int precision, const delta_meshes &m, const int32_t *pa,
                        const int32_t *pb, int64_t n_pairs, const delta_contacts *out, int64_t *n_out,
                        delta_stats *stats, int64_t *counters = nullptr, const Pose *pose = nullptr);

// Resident blocks per SM of a culled driver's two kernels (the culling kernel and the
// survivors' solver): the largest caps delta_ctx::cull_blocks_per_sm / surv_blocks_per_sm
// can take (detect.cu).
cudaError_t detect_launch_limits(int driver, int *cull_per_sm, int *surv_per_sm);

// Fixed-capacity (graph-capturable) detection (detect.cu).  `pose`: as for detect_run
// (null: the certified driver reads the meshes' vertices and culls without body boxes).
// `tri_bits`: bits of a triangle index within a body (every body has
// fewer than 2^tri_bits triangles), used to pack the contact sort keys.
size_t detect_fixed_temp_bytes(int64_t pair_cap, int64_t cap);
size_t detect_fixed_state_bytes(int64_t pair_cap, int64_t cap);
// Fills the identity permutation of a freshly allocated fixed-capacity state (once).
delta_status detect_fixed_init(cudaStream_t s, void *state, int64_t pair_cap, int64_t cap);
delta_status detect_run_fixed(delta_ctx *ctx, cudaStream_t s, int driver, const delta_meshes &m, const int32_t *pa,
                              const int32_t *pb, int64_t pair_cap, const delta_contacts &out, int64_t *d_ncontacts,
                              int *d_ovf, int ovf_code, int64_t *d_counters, int64_t *d_count_log, void *state,
                              void *temp, size_t temp_bytes, const Pose *pose = nullptr, int tri_bits = 16);

// Thread-local last-error text (capi.cu).
delta_status set_error(delta_status st, const std::string &msg);
delta_status cuda_error(cudaError_t e, const char *where);

}  // namespace delta

// Device buffer owned by a context; grows on demand, never shrinks.
struct delta_buffer {
  void *ptr = nullptr;
  size_t bytes = 0;
};

struct delta_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int64_t launches = 0;
  // launch shapes of the pair kernels [method][precision], set by autotuning
  delta::PairLaunch pair_launch[6][2];
  bool pair_launch_set[6][2] = {};
  delta_buffer scratch[32];
  // host-buffer entry points: copy streams and per-chunk events of the pipelined transfers
  cudaStream_t copy_in = nullptr, copy_out = nullptr;
  cudaEvent_t events[3 * 16] = {};
  int mlp_engine = DELTA_MLP_TCGEN05;  // network engine of the learned hybrid and its training GEMM
  int *gemm_err = nullptr;             // device flag: a tcgen05 GEMM's bounded wait gave up
  // launch shapes of the culled drivers' kernels (blocks per SM; 0 = as many as fit), set
  // by delta_sim_autotune
  int cull_blocks_per_sm = 0, surv_blocks_per_sm = 0;
  int64_t launch_epoch = 0;  // bumped when they change: recorded graphs are recorded again
  void *pinned = nullptr;
  size_t pinned_bytes = 0;
};

namespace delta {
// Launch shape of the pair kernel of (method, precision) on this context: the one set by
// delta_set_pair_launch / delta_autotune_pairs, else the default.
inline PairLaunch ctx_pair_launch(const delta_ctx *ctx, int method, int precision) {
  return ctx->pair_launch_set[method][precision] ? ctx->pair_launch[method][precision] : default_pair_launch(method);
}
// Host-buffer pipeline: stages the pair list (a, b: 9 planes of ld doubles) through the
// device in chunks, H2D on one copy stream, `run` on the context stream, D2H of p, q, dist
// (and flags when given) on another, so transfers of neighbouring chunks overlap the
// compute.  `run(c0, nc, da, db, ldd, dp, dq, dd, df)` enqueues chunk [c0, c0+nc) on the
// context stream (device planes of pitch ldd); `after(k)` (optional) enqueues per-chunk
// bookkeeping after it.  Synchronises.
delta_status host_pipeline(
    delta_ctx *ctx, int64_t n, const double *a, const double *b, int64_t ld, double *p, double *q, double *dist,
    uint8_t *flags,
    const std::function<delta_status(int64_t, int64_t, const double *, const double *, int64_t, double *, double *,
                                     double *, uint8_t *)> &run,
    const std::function<delta_status(int)> &after = nullptr);
// Returns a device buffer of at least `bytes` in slot `slot` of the context.
delta_status ctx_scratch(delta_ctx *ctx, int slot, size_t bytes, void **out);
delta_status ctx_pinned(delta_ctx *ctx, size_t bytes, void **out);
}  // namespace delta
