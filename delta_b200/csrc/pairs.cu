// pairs.cu -- pair-list narrowphase kernels (one thread per triangle pair).
//
// Input planes a[9*ld], b[9*ld] (plane 3*vertex+coord), outputs p[3*ld], q[3*ld],
// dist[n], flags[n].  Every warp reads 18 consecutive 256-byte segments, one per plane,
// and writes 7 more, so the loads and stores are fully coalesced.  Replaces the
// per-pair loops of bf()/penalty() (bf.cpp:95-118, penalty.cpp:187-210) and the SIMD
// pair-list kernels ispc_bf / ispc_pen (bf.ispc:3, penalty.ispc:154).
#include "internal.h"
#include "tri_cert.cuh"
#include "tri_gjk.cuh"
#include "tri_ref.cuh"

namespace delta {

enum { M_BF = 0, M_PENALTY = 1, M_PENALTY_ITER = 2, M_GJK = 3, M_HYBRID_PAIR = 4, M_BF_CERT = 5 };

// Launch bounds of the pair kernel: the FP64 bfSolver kernel is held to 96 registers (5
// blocks of 128 per SM; 109 unbounded, with one 256-thread block fewer per SM), the
// others keep their registers.
template <class R, int M>
struct PairBounds {
  static constexpr int kThreads = 256, kMinBlocks = 1;
};
template <>
struct PairBounds<xf64, M_BF> {
  static constexpr int kThreads = 128, kMinBlocks = 5;
};

// A warp walks the list 32 pairs at a time and meets at __syncwarp after each group: the
// lanes of a divergent solver would otherwise drift apart over the iterations of a
// grid-stride loop and run as several partial warps (measured: 4x slower when each
// thread takes ~50 pairs).
template <class R, int M>
__global__ void __launch_bounds__(PairBounds<R, M>::kThreads, PairBounds<R, M>::kMinBlocks)
    k_pairs(int64_t n, const double *__restrict__ a, const double *__restrict__ b, int64_t ld, double max_error,
            double *__restrict__ p, double *__restrict__ q, double *__restrict__ dist, uint8_t *__restrict__ flags) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
    const int64_t i = base + lane;
    if (i >= n) {
      __syncwarp();
      continue;
    }
    R A[3][3], B[3][3];
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        A[v][k] = from_f64<R>(__ldg(a + (3 * v + k) * ld + i));
        B[v][k] = from_f64<R>(__ldg(b + (3 * v + k) * ld + i));
      }
    R pq[6];
    int flag = 0;
    const R me = from_f64<R>(max_error);
    if constexpr (M == M_BF) {
      bf_solve_lean(A, B, pq);
    } else if constexpr (M == M_PENALTY) {
      penalty_ref(A, B, me, false, pq, flag);
    } else if constexpr (M == M_PENALTY_ITER) {
      penalty_ref(A, B, me, true, pq, flag);
    } else if constexpr (M == M_GJK) {
      gjk_ref(A, B, pq);
    } else {  // per-pair hybrid: penalty, bf when the pair reports failure
      penalty_ref(A, B, me, false, pq, flag);
      if (flag) bf_solve_lean(A, B, pq);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      p[k * ld + i] = to_f64(pq[k]);
      q[k * ld + i] = to_f64(pq[3 + k]);
    }
    dist[i] = to_f64(pq_distance(pq));
    if (flags) flags[i] = (uint8_t)flag;
    __syncwarp();
  }
}

// bf_cert: warps walk the pair list 32 pairs at a time (the certificate's candidate queue
// is shared by the warp).
template <int W>
__global__ void __launch_bounds__(32 * W) k_pairs_cert(int64_t n, const double *__restrict__ a,
                                                       const double *__restrict__ b, int64_t ld,
                                                       double *__restrict__ p, double *__restrict__ q,
                                                       double *__restrict__ dist, uint8_t *__restrict__ flags) {
  __shared__ CertWarpSmem sm[W];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t base = ((int64_t)blockIdx.x * (blockDim.x >> 5) + warp) * 32; base < n; base += nwarps * 32) {
    const int64_t i = base + lane;
    const bool valid = i < n;
    const int64_t ii = valid ? i : n - 1;
    double A[3][3], B[3][3];
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        A[v][k] = __ldg(a + (3 * v + k) * ld + ii);
        B[v][k] = __ldg(b + (3 * v + k) * ld + ii);
      }
    double out[6];
    const int evals = bf_cert_warp(A, B, valid, out, sm[warp]);
    if (valid) {
      xf64 pq[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) pq[k] = xf64(out[k]);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        p[k * ld + i] = out[k];
        q[k * ld + i] = out[3 + k];
      }
      dist[i] = pq_distance(pq).v;
      if (flags) flags[i] = (uint8_t)evals;
    }
  }
}

// The certified kernel over an index list: pairs idx[0 .. *count) of the pair list (the
// count is read on the device, so the list can be built by an earlier kernel on the
// stream without a host round trip).  With `stage`, entry j's coordinates are read from
// stage[stage_at(j, c)] (a's 9, then b's; one contiguous tile per warp) instead of being
// gathered from a and b; results go to pair idx[j] of p, q, dist.
template <int W>
__global__ void __launch_bounds__(32 * W) k_pairs_cert_indexed(const uint32_t *__restrict__ count,
                                                               const uint32_t *__restrict__ idx,
                                                               const double *__restrict__ a,
                                                               const double *__restrict__ b, int64_t ld,
                                                               const double *__restrict__ stage,
                                                               double *__restrict__ p, double *__restrict__ q,
                                                               double *__restrict__ dist) {
  __shared__ CertWarpSmem sm[W];
  const int64_t n = *count;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t base = ((int64_t)blockIdx.x * (blockDim.x >> 5) + warp) * 32; base < n; base += nwarps * 32) {
    const bool valid = base + lane < n;
    const int64_t j = valid ? base + lane : n - 1;
    const int64_t i = idx[j];
    double A[3][3], B[3][3];
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        A[v][k] = stage ? __ldg(stage + stage_at(j, 3 * v + k)) : __ldg(a + (3 * v + k) * ld + i);
        B[v][k] = stage ? __ldg(stage + stage_at(j, 9 + 3 * v + k)) : __ldg(b + (3 * v + k) * ld + i);
      }
    double out[6];
    bf_cert_warp(A, B, valid, out, sm[warp]);
    if (valid) {
      xf64 pq[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) pq[k] = xf64(out[k]);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        p[k * ld + i] = out[k];
        q[k * ld + i] = out[3 + k];
      }
      dist[i] = pq_distance(pq).v;
    }
  }
}

// cfg.blocks_per_sm > 0 caps the grid at that many blocks per SM (a grid-stride loop);
// 0 launches one thread per pair
template <class R, int M>
static cudaError_t launch_one(cudaStream_t s, int64_t n, const double *a, const double *b, int64_t ld, double me,
                              double *p, double *q, double *dist, uint8_t *flags, PairLaunch cfg) {
  int threads = cfg.threads == 64 || cfg.threads == 128 ? cfg.threads : 256;
  if (threads > PairBounds<R, M>::kThreads) threads = PairBounds<R, M>::kThreads;
  int64_t blocks = (n + threads - 1) / threads;
  if (cfg.blocks_per_sm > 0 && blocks > (int64_t)kNumSMs * cfg.blocks_per_sm) blocks = (int64_t)kNumSMs * cfg.blocks_per_sm;
  if (blocks > 0x7fffffffLL) blocks = 0x7fffffffLL;
  if (blocks < 1) blocks = 1;
  k_pairs<R, M><<<(unsigned)blocks, threads, 0, s>>>(n, a, b, ld, me, p, q, dist, flags);
  return cudaGetLastError();
}

template <class R>
static cudaError_t launch_prec(int method, cudaStream_t s, int64_t n, const double *a, const double *b, int64_t ld,
                               double me, double *p, double *q, double *dist, uint8_t *flags, PairLaunch cfg) {
  switch (method) {
    case M_BF: return launch_one<R, M_BF>(s, n, a, b, ld, me, p, q, dist, flags, cfg);
    case M_PENALTY: return launch_one<R, M_PENALTY>(s, n, a, b, ld, me, p, q, dist, flags, cfg);
    case M_PENALTY_ITER: return launch_one<R, M_PENALTY_ITER>(s, n, a, b, ld, me, p, q, dist, flags, cfg);
    case M_GJK: return launch_one<R, M_GJK>(s, n, a, b, ld, me, p, q, dist, flags, cfg);
    case M_HYBRID_PAIR: return launch_one<R, M_HYBRID_PAIR>(s, n, a, b, ld, me, p, q, dist, flags, cfg);
    default: return cudaErrorInvalidValue;
  }
}

template <int W>
static cudaError_t launch_cert(cudaStream_t s, int64_t n, const double *a, const double *b, int64_t ld, double *p,
                               double *q, double *dist, uint8_t *flags, PairLaunch cfg) {
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pairs_cert<W>, 32 * W, 0);
  if (e != cudaSuccess) return e;
  int64_t blocks = (n + 32 * W - 1) / (32 * W);
  const int64_t per = cfg.blocks_per_sm > 0 ? cfg.blocks_per_sm : 8;
  const int64_t cap = (int64_t)kNumSMs * (per_sm > 0 ? per_sm : 1) * per;
  if (blocks > cap) blocks = cap;
  k_pairs_cert<W><<<(unsigned)(blocks > 0 ? blocks : 1), 32 * W, 0, s>>>(n, a, b, ld, p, q, dist, flags);
  return cudaGetLastError();
}

int pair_max_threads(int method, int precision) {
  if (method == M_BF_CERT) return 128;
  return (method == M_BF && precision == 0) ? PairBounds<xf64, M_BF>::kThreads : 256;
}

cudaError_t launch_pairs_cfg(int method, int precision, cudaStream_t s, int64_t n, const double *a, const double *b,
                             int64_t ld, double max_error, double *p, double *q, double *dist, uint8_t *flags,
                             PairLaunch cfg) {
  if (method == M_BF_CERT) {
    if (cfg.threads == 64) return launch_cert<2>(s, n, a, b, ld, p, q, dist, flags, cfg);
    return launch_cert<4>(s, n, a, b, ld, p, q, dist, flags, cfg);
  }
  if (precision == 0) return launch_prec<xf64>(method, s, n, a, b, ld, max_error, p, q, dist, flags, cfg);
  return launch_prec<float>(method, s, n, a, b, ld, max_error, p, q, dist, flags, cfg);
}

cudaError_t launch_cert_indexed(cudaStream_t s, const uint32_t *count, int64_t max_count, const uint32_t *idx,
                                const double *a, const double *b, int64_t ld, double *p, double *q, double *dist,
                                PairLaunch cfg, const double *stage) {
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pairs_cert_indexed<4>, 128, 0);
  if (e != cudaSuccess) return e;
  int64_t blocks = (max_count + 127) / 128;
  const int64_t per = cfg.blocks_per_sm > 0 ? cfg.blocks_per_sm : 8;
  const int64_t cap = (int64_t)kNumSMs * (per_sm > 0 ? per_sm : 1) * per;
  if (blocks > cap) blocks = cap;
  k_pairs_cert_indexed<4><<<(unsigned)(blocks > 0 ? blocks : 1), 128, 0, s>>>(count, idx, a, b, ld, stage, p, q, dist);
  return cudaGetLastError();
}

cudaError_t launch_pairs(int method, int precision, cudaStream_t s, int64_t n, const double *a, const double *b,
                         int64_t ld, double max_error, double *p, double *q, double *dist, uint8_t *flags) {
  return launch_pairs_cfg(method, precision, s, n, a, b, ld, max_error, p, q, dist, flags, default_pair_launch(method));
}

}  // namespace delta
