// detect.cu -- particle-pair narrowphase drivers (bf, penalty, hybrids, gjk, stat variants).
//
// Work unit: one row = one triangle of body A against all triangles of body B of a
// candidate pair, processed by one warp (lane l handles B triangles l, l+32, ...).  Rows
// are handed out by a persistent work queue (an atomic row counter), so candidate pairs
// of very different sizes share the SMs evenly.  The row-level decisions of the hybrid
// drivers (hybrid.cpp:151-170, 434-460) and the row minimum of the stat drivers
// (hybrid.cpp:605-617) are warp reductions.  Contacts are appended with one atomic per
// warp and a 64-bit key (pair, A triangle, B triangle); a radix sort by key then
// restores the serial order of the reference drivers, so the output is deterministic.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdlib>

#include "pdl.cuh"
#include "blockscan.cuh"
#include "internal.h"
#include "pose.cuh"
#include "tri_cert.cuh"
#include "tri_learned.cuh"
#include "tri_gjk.cuh"
#include "tri_ref.cuh"

namespace delta {

namespace {

constexpr unsigned kFull = 0xffffffffu;

struct RawContacts {
  double *f;        // 14 planes of cap: x(3) normal(3) depth P(3) Q(3) eps_total
  int32_t *i;       // 4 planes: master slave tri_a tri_b
  uint8_t *fric;
  uint64_t *key;
  int64_t cap;
  unsigned long long *count;
  // certified driver: triangle pairs that survive the box test, as keys (pair, A tri, B tri)
  uint64_t *sv;
  int64_t sv_cap;
  unsigned long long *sv_count;
  // certified driver: per-body boxes (lo[3], hi[3]) for the culling, or null
  const double *bbox;
  // certified driver: with pose.rx set, the vertices are formed from the bodies' poses (the
  // mesh arrays are not current) and the body boxes come from pose_box
  Pose pose;
  // sort key of a contact: pair << 2 tbits | A triangle << tbits | B triangle
  int tbits;
  // fixed-capacity certified driver: contacts counted per pair (pcnt, zeroed by the culling)
  // and each contact's rank of arrival within its pair (slot), for the sort-free ordering;
  // null elsewhere
  unsigned long long *pcnt;
  uint32_t *slot;
  // culled drivers: the body-pair work queue of the culling kernel (zeroed before it runs);
  // null: blocks take the pairs by a fixed stride
  unsigned long long *pair_queue;
};

struct DevStats {
  unsigned long long hist[17];
  unsigned long long penalty_fails, batch_fails, batch_size;
  double batch_error;
  unsigned long long tri_pairs, evaluated;  // sum of nA*nB; pairs the solver ran on
};

struct RowCtx {
  int64_t k;       // pair index
  int32_t iA;      // triangle of A (within the body)
  int64_t tA, tB0; // global triangle indices
  int32_t nB;
  double epsA, epsB;
  int32_t idA, idB;
  uint8_t fric;
};

template <class R>
__device__ __forceinline__ void load_tri(const delta_meshes &m, int64_t t, R T[3][3]) {
#pragma unroll
  for (int v = 0; v < 3; ++v) {
    T[v][0] = from_f64<R>(__ldg(m.x + 3 * t + v));
    T[v][1] = from_f64<R>(__ldg(m.y + 3 * t + v));
    T[v][2] = from_f64<R>(__ldg(m.z + 3 * t + v));
  }
}

__device__ __forceinline__ void load_tri64(const delta_meshes &m, int64_t t, double T[3][3]) {
#pragma unroll
  for (int v = 0; v < 3; ++v) {
    T[v][0] = __ldg(m.x + 3 * t + v);
    T[v][1] = __ldg(m.y + 3 * t + v);
    T[v][2] = __ldg(m.z + 3 * t + v);
  }
}

// Triangle t of body `body`, current vertices: formed from the pose when one is given and
// the body moves, read from the meshes otherwise.
__device__ __forceinline__ void load_tri_cur(const delta_meshes &m, const Pose &P, int32_t body, int64_t t,
                                             double T[3][3]) {
  if (P.rx && !P.obstacle[body]) posed_tri(P, body_pose(P, body), t, T);
  else load_tri64(m, t, T);
}

// The per-triangle-pair solver of each driver.  Returns closest points (FP64 values).
enum Solver { S_BF, S_PENALTY, S_PENALTY_ITER, S_GJK };

template <class R, int S>
__device__ __forceinline__ void solve(const delta_meshes &m, int64_t tA, int64_t tB, double max_err, double pq[6],
                                      int &flag) {
  {
    R A[3][3], B[3][3], out[6];
    load_tri<R>(m, tA, A);
    load_tri<R>(m, tB, B);
    if constexpr (S == S_BF) bf_solve_lean(A, B, out);
    else if constexpr (S == S_PENALTY) penalty_ref(A, B, from_f64<R>(max_err), false, out, flag);
    else if constexpr (S == S_PENALTY_ITER) penalty_ref(A, B, from_f64<R>(max_err), true, out, flag);
    else gjk_ref(A, B, out);
#pragma unroll
    for (int k = 0; k < 6; ++k) pq[k] = to_f64(out[k]);
  }
}

// d = |P_B - P_A| (bf.cpp:117) in FP64 reference arithmetic
__device__ __forceinline__ double pq_dist64(const double pq[6]) {
  xf64 x[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) x[k] = xf64(pq[k]);
  return pq_distance(x).v;
}

// contactpoint(PA, epsA, idA, QB, epsB, idB, friction), contactpoint.cpp:116-155
__device__ __forceinline__ void write_contact(const RawContacts &rc, int64_t pos, const double pq[6], const RowCtx &r,
                                              int32_t tb) {
  const int64_t cap = rc.cap;
  xf64 P[3] = {xf64(pq[0]), xf64(pq[1]), xf64(pq[2])}, Q[3] = {xf64(pq[3]), xf64(pq[4]), xf64(pq[5])};
  const xf64 two = xf64(2.0);
  const xf64 eps_total = xf64(r.epsA) + xf64(r.epsB);
  const xf64 dist = sqrt_(((Q[0] - P[0]) * (Q[0] - P[0])) + ((Q[1] - P[1]) * (Q[1] - P[1])) +
                          ((Q[2] - P[2]) * (Q[2] - P[2])));
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    rc.f[(0 + k) * cap + pos] = ((P[k] + Q[k]) / two).v;
    rc.f[(3 + k) * cap + pos] = ((P[k] - Q[k]) / dist).v;
    rc.f[(7 + k) * cap + pos] = P[k].v;
    rc.f[(10 + k) * cap + pos] = Q[k].v;
  }
  rc.f[6 * cap + pos] = (eps_total - dist).v;
  rc.f[13 * cap + pos] = eps_total.v;
  rc.i[0 * cap + pos] = r.idA;
  rc.i[1 * cap + pos] = r.idB;
  rc.i[2 * cap + pos] = r.iA;
  rc.i[3 * cap + pos] = tb;
  rc.fric[pos] = r.fric;
  rc.key[pos] = ((uint64_t)r.k << (2 * rc.tbits)) | ((uint64_t)r.iA << rc.tbits) | (uint64_t)tb;
}

// Slot for the calling lane in an append buffer: one atomic per group of lanes that
// arrive together (__activemask), whatever the warp's convergence after the
// data-dependent solver branches before the call.
__device__ __forceinline__ int64_t agg_slot(unsigned long long *count) {
  const unsigned grp = __activemask();
  const int lane = threadIdx.x & 31, leader = __ffs(grp) - 1;
  unsigned long long base = 0;
  if (lane == leader) base = atomicAdd(count, (unsigned long long)__popc(grp));
  base = __shfl_sync(grp, base, leader);
  return (int64_t)base + __popc(grp & ((1u << lane) - 1u));
}

// Append of the lanes with `take` set (their order is irrelevant: the key sort fixes the
// final order).
__device__ __forceinline__ void emit(const RawContacts &rc, bool take, const double pq[6], const RowCtx &r, int32_t tb) {
  if (!take) return;
  const int64_t pos = agg_slot(rc.count);
  if (pos < rc.cap) {
    write_contact(rc, pos, pq, r, tb);
    if (rc.pcnt) rc.slot[pos] = (uint32_t)atomicAdd(rc.pcnt + r.k, 1ull);
  }
}

__device__ __forceinline__ int warp_sum(int v) { return __reduce_add_sync(kFull, v); }

__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(kFull, v, o));
  return v;
}

// Applies `fn(tb, valid)` to the row's B triangles in chunks of 32 (all lanes take part).
template <class F>
__device__ __forceinline__ void for_row(int32_t nB, F &&fn) {
  const int lane = threadIdx.x & 31;
  for (int32_t base = 0; base < nB; base += 32) {
    const int32_t tb = base + lane;
    fn(tb, tb < nB);
  }
}

template <class R, int DRV>
__device__ void process_row(const delta_meshes &m, const RowCtx &r, const RawContacts &rc, DevStats *st) {
  const xf64 margin = xf64(r.epsA) + xf64(r.epsB);
  const double max_err = (margin / xf64(16.0)).v;  // (epsA+epsB)/16, hybrid.cpp:60
  const double mg = margin.v;
  double pq[6];
  int flag = 0;
  if constexpr (DRV == DELTA_DRV_BF || DRV == DELTA_DRV_GJK) {
    constexpr int S = DRV == DELTA_DRV_BF ? S_BF : S_GJK;
    for_row(r.nB, [&](int32_t tb, bool valid) {
      bool take = false;
      if (valid) {
        solve<R, S>(m, r.tA, r.tB0 + tb, max_err, pq, flag);
        take = pq_dist64(pq) <= mg;  // bf.cpp:125
      }
      emit(rc, take, pq, r, tb);
    });
  } else if constexpr (DRV == DELTA_DRV_PENALTY) {
    for_row(r.nB, [&](int32_t tb, bool valid) {
      bool take = false;
      if (valid) {
        solve<R, S_PENALTY>(m, r.tA, r.tB0 + tb, max_err, pq, flag);
        take = pq_dist64(pq) < mg;  // penalty.cpp:217
      }
      emit(rc, take, pq, r, tb);
    });
  } else if constexpr (DRV == DELTA_DRV_PENALTY_STAT) {
    for_row(r.nB, [&](int32_t tb, bool valid) {
      int it = 0;  // penalty.cpp:86
      bool take = false;
      if (valid) {
        solve<R, S_PENALTY_ITER>(m, r.tA, r.tB0 + tb, max_err, pq, it);
        // penalty.cpp:96 scans coordinate indices below nB: triangles tb with 3*tb < nB
        take = (3 * tb < r.nB) && pq_dist64(pq) <= mg;
      }
      if (valid && it >= 0 && it < 17) atomicAdd(&st->hist[it], 1ull);
      emit(rc, take, pq, r, tb);
    });
  } else {
    // hybrids: penalty over the row, count failures, decide the fallback for the row
    int fails = 0;
    for_row(r.nB, [&](int32_t tb, bool valid) {
      int f = 0;
      if (valid) solve<R, S_PENALTY>(m, r.tA, r.tB0 + tb, max_err, pq, f);
      fails += f;
    });
    const int counter = warp_sum(fails);
    bool rerun;
    const xf64 me = xf64(max_err);
    if constexpr (DRV == DELTA_DRV_HYBRID_TRIANGLE) {
      rerun = counter > 0;  // hybrid.cpp:151-156
    } else if constexpr (DRV == DELTA_DRV_HYBRID_BATCH) {
      rerun = (xf64((double)counter) * me) > ((me * xf64((double)(3 * (int64_t)r.nB))) / xf64(32.0));  // :434-440
    } else {
      rerun = (xf64((double)counter) * me) > ((me * xf64((double)r.nB)) / xf64(32.0));  // :565-573
      if ((threadIdx.x & 31) == 0) {
        atomicAdd(&st->batch_size, (unsigned long long)r.nB);
        atomicAdd(&st->batch_error, max_err);
        atomicAdd(&st->penalty_fails, (unsigned long long)counter);
        if (rerun) atomicAdd(&st->batch_fails, 1ull);
      }
    }
    auto final_solve = [&](int32_t tb) {
      int f = 0;
      if (rerun) solve<R, S_BF>(m, r.tA, r.tB0 + tb, max_err, pq, f);
      else solve<R, S_PENALTY>(m, r.tA, r.tB0 + tb, max_err, pq, f);
    };
    if constexpr (DRV == DELTA_DRV_HYBRID_BATCH || DRV == DELTA_DRV_HYBRID_TRIANGLE) {
      for_row(r.nB, [&](int32_t tb, bool valid) {
        bool take = false;
        if (valid) {
          final_solve(tb);
          take = pq_dist64(pq) < mg;  // hybrid.cpp:176, 466
        }
        emit(rc, take, pq, r, tb);
      });
    } else {
      // stat variants keep only the row minimum (hybrid.cpp:319-326, 605-617)
      double mind = 1E99;
      for_row(r.nB, [&](int32_t tb, bool valid) {
        if (valid) {
          final_solve(tb);
          mind = fmin(mind, pq_dist64(pq));
        }
      });
      mind = warp_min(mind);
      for_row(r.nB, [&](int32_t tb, bool valid) {
        bool take = false;
        if (valid) {
          final_solve(tb);
          const double d = pq_dist64(pq);
          take = d <= mind && d < mg;
        }
        emit(rc, take, pq, r, tb);
      });
    }
  }
}

// per-body bounding boxes of the current vertices: one warp per body
__global__ void k_body_boxes(delta_meshes m, double *__restrict__ bbox) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t b = warp; b < m.n_bodies; b += nwarps) {
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t v = 3 * m.tri_offset[b] + lane; v < 3 * m.tri_offset[b + 1]; v += 32) {
      const double c[3] = {__ldg(m.x + v), __ldg(m.y + v), __ldg(m.z + v)};
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        lo[k] = fmin(lo[k], c[k]);
        hi[k] = fmax(hi[k], c[k]);
      }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      for (int o = 16; o > 0; o >>= 1) {
        lo[k] = fmin(lo[k], __shfl_xor_sync(kFull, lo[k], o));
        hi[k] = fmax(hi[k], __shfl_xor_sync(kFull, hi[k], o));
      }
    }
    if (lane == 0)
      for (int k = 0; k < 3; ++k) {
        bbox[6 * b + k] = lo[k];
        bbox[6 * b + 3 + k] = hi[k];
      }
  }
}

// Blocks of 128 per SM the driver kernel is bounded to: 5 (96 registers) for the FP64 bf
// driver, whose unbounded 134 registers left 3 (the same bound raised the FP64 pair
// kernel by 10%); the other drivers keep their registers.
template <class R, int DRV>
struct DetectBounds {
  static constexpr int kMinBlocks = 1;
};
template <>
struct DetectBounds<xf64, DELTA_DRV_BF> {
  static constexpr int kMinBlocks = 5;
};

template <class R, int DRV>
__global__ void __launch_bounds__(128, DetectBounds<R, DRV>::kMinBlocks) k_detect(delta_meshes m, const int32_t *__restrict__ pa,
                                                const int32_t *__restrict__ pb,
                                                const int64_t *__restrict__ row_offset, int64_t n_pairs,
                                                const int64_t *total_rows_p, RawContacts rc, DevStats *st,
                                                unsigned long long *queue) {
  const int lane = threadIdx.x & 31;
  const int64_t total_rows = *total_rows_p;
  for (;;) {
    unsigned long long row = 0;
    if (lane == 0) row = atomicAdd(queue, 1ull);
    row = __shfl_sync(kFull, row, 0);
    if ((int64_t)row >= total_rows) return;
    // pair k: last k with row_offset[k] <= row
    int64_t lo = 0, hi = n_pairs;
    while (hi - lo > 1) {
      const int64_t mid = (lo + hi) >> 1;
      if (row_offset[mid] <= (int64_t)row) lo = mid;
      else hi = mid;
    }
    RowCtx r;
    r.k = lo;
    const int32_t a = pa[lo], b = pb[lo];
    r.iA = (int32_t)((int64_t)row - row_offset[lo]);
    r.tA = m.tri_offset[a] + r.iA;
    r.tB0 = m.tri_offset[b];
    r.nB = (int32_t)(m.tri_offset[b + 1] - r.tB0);
    r.epsA = m.eps[a];
    r.epsB = m.eps[b];
    r.idA = m.id[a];
    r.idB = m.id[b];
    r.fric = (m.friction[a] && m.friction[b]) ? 1 : 0;
    if (lane == 0) {
      atomicAdd(&st->tri_pairs, (unsigned long long)r.nB);
      atomicAdd(&st->evaluated, (unsigned long long)r.nB);
    }
    process_row<R, DRV>(m, r, rc, st);
  }
}

// ---- certified driver, phase 1: exact box culling, one block per particle pair ---------
// bf()'s distance is the length of a point pair on the two triangles, never below the gap
// between their bounding boxes, so a triangle pair whose boxes are farther apart than
// epsA+epsB (with a relative margin for rounding) cannot give a contact (bf.cpp:125).  A
// block stages in shared memory the A triangles whose box is within the cull distance of
// B's body box and the B triangles within it of A's body box (at most kCullList each;
// longer lists are taken in windows) and then tests the staged boxes pair by pair.  The
// survivors are exactly the triangle pairs whose boxes pass the test: every triangle box
// lies in its body box and the per-axis gaps, their squares and their sum are monotone in
// the boxes, so a triangle dropped against a body box fails against every triangle of
// that body too.
constexpr int kCullThreads = 128;
constexpr int kCullList = 256;
struct CullList {
  double lo[3][kCullList], hi[3][kCullList];
  uint16_t idx[kCullList];
  int n;
};

// squared gap between the boxes (alo, ahi) and (blo, bhi): the sum of the squares of the
// positive per-axis gaps
__device__ __forceinline__ double box_gap2(const double alo[3], const double ahi[3], const double blo[3],
                                           const double bhi[3]) {
  double g2 = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double g = fmax(blo[k] - ahi[k], alo[k] - bhi[k]);
    if (g > 0.0) g2 += g * g;
  }
  return g2;
}

// Stages the triangles cur, cur+1, ... of (t0, n) whose box lies within the cull distance
// of the box (olo, ohi) into L (in any order), kCullThreads at a time while L can take
// that many more; returns the cursor.  Called by the whole block.  With `q` (the body's
// pose, in shared memory) the vertices are formed from the reference vertices.
__device__ __forceinline__ int32_t cull_fill(const delta_meshes &m, const Pose &P, const BodyPose *q, int64_t t0,
                                             int32_t n, int32_t cur, const double olo[3], const double ohi[3],
                                             double cull2, CullList &L) {
  const int tid = threadIdx.x, lane = tid & 31;
  if (tid == 0) L.n = 0;
  __syncthreads();
  while (cur < n && L.n + kCullThreads <= kCullList) {
    const int32_t i = cur + tid;
    double lo[3] = {0.0, 0.0, 0.0}, hi[3] = {0.0, 0.0, 0.0};
    bool keep = false;
    if (i < n) {
      double T[3][3];
      if (q) posed_tri(P, *q, t0 + i, T);
      else load_tri64(m, t0 + i, T);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        lo[k] = fmin(T[0][k], fmin(T[1][k], T[2][k]));
        hi[k] = fmax(T[0][k], fmax(T[1][k], T[2][k]));
      }
      keep = box_gap2(lo, hi, olo, ohi) <= cull2;
    }
    const unsigned bal = __ballot_sync(kFull, keep);
    int base = 0;
    if (lane == 0 && bal) base = atomicAdd(&L.n, __popc(bal));
    base = __shfl_sync(kFull, base, 0);
    if (keep) {
      const int s = base + __popc(bal & ((1u << lane) - 1u));
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        L.lo[k][s] = lo[k];
        L.hi[k][s] = hi[k];
      }
      L.idx[s] = (uint16_t)i;
    }
    cur += kCullThreads;
    __syncthreads();
  }
  return cur;
}

// Pairs k = block, block + n_blocks, ... (entries with a negative body are empty).
// Survivor keys (pair << 32 | A triangle << 16 | B triangle) go to rc.sv; their order is
// free (the contacts are ordered by key afterwards).  With rc.pose the vertices are formed
// from the bodies' poses and the body boxes come from pose_box; otherwise rc.bbox holds
// the body boxes of the current vertices (null: no body-box tests).
__global__ void __launch_bounds__(kCullThreads, 8) k_cull_pairs(delta_meshes m, const int32_t *__restrict__ pa,
                                                             const int32_t *__restrict__ pb, int64_t n_pairs,
                                                             RawContacts rc, DevStats *st) {
  dep_sync();
  __shared__ CullList LA, LB;
  __shared__ BodyPose QA, QB;
  __shared__ int64_t s_next;
  const int tid = threadIdx.x;
  if (rc.pcnt && blockIdx.x == 0 && tid == 0) rc.pcnt[n_pairs] = 0;
  // a persistent work queue of body pairs: each block takes the next pair when it is done
  // with its last, so uneven pairs (a wall of thousands of triangles next to small meshes)
  // do not leave the other blocks idle; without a queue, a fixed stride
  int64_t k = blockIdx.x;
  if (rc.pair_queue) {
    if (tid == 0) s_next = (int64_t)atomicAdd(rc.pair_queue, 1ull);
    __syncthreads();
    k = s_next;
  }
  while (k < n_pairs) {
    do {  // one body pair; `continue` ends it
    if (rc.pcnt && tid == 0) rc.pcnt[k] = 0;  // the pair's contact count (k_cert_survivors)
    const int32_t a = pa[k], b = pb[k];
    if (a < 0 || b < 0) continue;
    const int64_t tA0 = m.tri_offset[a], tB0 = m.tri_offset[b];
    const int32_t nA = (int32_t)(m.tri_offset[a + 1] - tA0), nB = (int32_t)(m.tri_offset[b + 1] - tB0);
    if (tid == 0) atomicAdd(&st->tri_pairs, (unsigned long long)nA * (unsigned long long)nB);
    const double mg = (xf64(m.eps[a]) + xf64(m.eps[b])).v;
    const double cull = mg * (1.0 + 1e-9) + 1e-12, cull2 = cull * cull;
    double Alo[3], Ahi[3], Blo[3], Bhi[3];
    const Pose &P = rc.pose;
    if (P.rx) {
      pose_box(P, a, Alo, Ahi);
      pose_box(P, b, Blo, Bhi);
    } else {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        Alo[c] = rc.bbox ? rc.bbox[6 * (int64_t)a + c] : -INFINITY;
        Ahi[c] = rc.bbox ? rc.bbox[6 * (int64_t)a + 3 + c] : INFINITY;
        Blo[c] = rc.bbox ? rc.bbox[6 * (int64_t)b + c] : -INFINITY;
        Bhi[c] = rc.bbox ? rc.bbox[6 * (int64_t)b + 3 + c] : INFINITY;
      }
    }
    if (box_gap2(Alo, Ahi, Blo, Bhi) > cull2) continue;
    const bool moveA = P.rx && !P.obstacle[a], moveB = P.rx && !P.obstacle[b];
    if (tid == 0 && moveA) QA = body_pose(P, a);
    if (tid == 1 && moveB) QB = body_pose(P, b);
    __syncthreads();  // the poses are read by cull_fill (which synchronises before refilling)
    for (int32_t cb = 0; cb < nB;) {
      cb = cull_fill(m, P, moveB ? &QB : nullptr, tB0, nB, cb, Alo, Ahi, cull2, LB);
      const int nLB = LB.n;
      if (nLB == 0) continue;
      for (int32_t ca = 0; ca < nA;) {
        ca = cull_fill(m, P, moveA ? &QA : nullptr, tA0, nA, ca, Blo, Bhi, cull2, LA);
        const int np = LA.n * nLB;
        for (int j = tid; j < np; j += kCullThreads) {
          const int ia = j / nLB, ib = j - ia * nLB;
          const double alo[3] = {LA.lo[0][ia], LA.lo[1][ia], LA.lo[2][ia]};
          const double ahi[3] = {LA.hi[0][ia], LA.hi[1][ia], LA.hi[2][ia]};
          const double blo[3] = {LB.lo[0][ib], LB.lo[1][ib], LB.lo[2][ib]};
          const double bhi[3] = {LB.hi[0][ib], LB.hi[1][ib], LB.hi[2][ib]};
          if (box_gap2(alo, ahi, blo, bhi) <= cull2) {
            const int64_t pos = agg_slot(rc.sv_count);
            if (pos < rc.sv_cap)
              rc.sv[pos] = ((uint64_t)k << 32) | ((uint64_t)LA.idx[ia] << 16) | (uint64_t)LB.idx[ib];
          }
        }
        __syncthreads();  // LA is refilled next
      }
    }
    } while (0);
    if (rc.pair_queue) {
      __syncthreads();  // every thread has read s_next for this pair
      if (tid == 0) s_next = (int64_t)atomicAdd(rc.pair_queue, 1ull);
      __syncthreads();
      k = s_next;
    } else {
      k += gridDim.x;
    }
  }
}

// DELTA_CULL_STRIDE=1 in the environment: the culling kernel's blocks take the body pairs
// by a fixed stride instead of the work queue (for comparison).
inline bool cull_stride() {
  static const bool v = [] {
    const char *e = std::getenv("DELTA_CULL_STRIDE");
    return e && e[0] == '1';
  }();
  return v;
}

// cap: blocks per SM (the time-step autotuner's choice), 0 = as many as fit
inline cudaError_t launch_cull(cudaStream_t s, const delta_meshes &m, const int32_t *pa, const int32_t *pb,
                               int64_t n_pairs, const RawContacts &rc, DevStats *st, int cap = 0, bool dep = false) {
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cull_pairs, kCullThreads, 0);
  if (e != cudaSuccess) return e;
  if (cap > 0 && cap < per_sm) per_sm = cap;
  int64_t blocks = (int64_t)kNumSMs * (per_sm > 0 ? per_sm : 1);
  if (blocks > n_pairs) blocks = n_pairs > 0 ? n_pairs : 1;
  return launch_dep(dep, k_cull_pairs, (unsigned)blocks, kCullThreads, 0, s, m, pa, pb, n_pairs, rc, st);
}

// Certified bf over the survivors of the box test, 32 per warp (any mix of pairs).
__global__ void __launch_bounds__(128, 5) k_cert_survivors(delta_meshes m, const int32_t *__restrict__ pa,
                                                        const int32_t *__restrict__ pb, RawContacts rc,
                                                        DevStats *st) {
  dep_sync();
  __shared__ CertWarpSmem sm[4];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned long long cnt = *rc.sv_count;
  const int64_t n = (int64_t)cnt < rc.sv_cap ? (int64_t)cnt : rc.sv_cap;
  if (n == 0) return;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t base = ((int64_t)blockIdx.x * (blockDim.x >> 5) + warp) * 32; base < n; base += nwarps * 32) {
    const int64_t i = base + lane;
    const bool valid = i < n;
    const uint64_t key = rc.sv[valid ? i : n - 1];
    RowCtx r;
    r.k = (int64_t)(key >> 32);
    r.iA = (int32_t)((key >> 16) & 0xffff);
    const int32_t tb = (int32_t)(key & 0xffff);
    const int32_t a = pa[r.k], b = pb[r.k];
    r.tA = m.tri_offset[a] + r.iA;
    r.tB0 = m.tri_offset[b];
    r.epsA = m.eps[a];
    r.epsB = m.eps[b];
    r.idA = m.id[a];
    r.idB = m.id[b];
    r.fric = (m.friction[a] && m.friction[b]) ? 1 : 0;
    double A[3][3], B[3][3], pq[6];
    load_tri_cur(m, rc.pose, a, r.tA, A);
    load_tri_cur(m, rc.pose, b, r.tB0 + tb, B);
    bf_cert_warp(A, B, valid, pq, sm[warp]);
    const double mg = (xf64(r.epsA) + xf64(r.epsB)).v;
    const bool take = valid && pq_dist64(pq) <= mg;  // bf.cpp:125
    emit(rc, take, pq, r, tb);
  }
}

// The reference's FP64 bfSolver (bf.cpp:217-1178, xf64) over the survivors of the box
// test, one per thread: the culled driver without the FP32 filter (DELTA_DRV_BF_CULLED),
// which separates what the culling gains from what the certified FP32 solver gains.
__global__ void __launch_bounds__(128, 5) k_bf64_survivors(delta_meshes m, const int32_t *__restrict__ pa,
                                                           const int32_t *__restrict__ pb, RawContacts rc) {
  dep_sync();
  const unsigned long long cnt = *rc.sv_count;
  const int64_t n = (int64_t)cnt < rc.sv_cap ? (int64_t)cnt : rc.sv_cap;
  // a warp takes 32 survivors at a time and meets at __syncwarp after them, so that its
  // lanes do not drift apart over the grid-stride loop (see k_pairs)
  const int lane = threadIdx.x & 31;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n;
       base += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = base + lane;
    if (i >= n) {
      __syncwarp();
      continue;
    }
    const uint64_t key = rc.sv[i];
    RowCtx r;
    r.k = (int64_t)(key >> 32);
    r.iA = (int32_t)((key >> 16) & 0xffff);
    const int32_t tb = (int32_t)(key & 0xffff);
    const int32_t a = pa[r.k], b = pb[r.k];
    r.tA = m.tri_offset[a] + r.iA;
    r.tB0 = m.tri_offset[b];
    r.epsA = m.eps[a];
    r.epsB = m.eps[b];
    r.idA = m.id[a];
    r.idB = m.id[b];
    r.fric = (m.friction[a] && m.friction[b]) ? 1 : 0;
    double A[3][3], B[3][3], pq[6];
    load_tri_cur(m, rc.pose, a, r.tA, A);
    load_tri_cur(m, rc.pose, b, r.tB0 + tb, B);
    xf64 A64[3][3], B64[3][3], out[6];
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        A64[v][k] = xf64(A[v][k]);
        B64[v][k] = xf64(B[v][k]);
      }
    bf_solve_lean(A64, B64, out);
#pragma unroll
    for (int k = 0; k < 6; ++k) pq[k] = out[k].v;
    const double mg = (xf64(r.epsA) + xf64(r.epsB)).v;
    emit(rc, pq_dist64(pq) <= mg, pq, r, tb);  // bf.cpp:125
    __syncwarp();
  }
}

// The learned FP32 hybrid over the survivors of the box test (DELTA_DRV_LEARNED), 32 per
// warp: each lane runs learned_pair_solve (2 FP32 projection sweeps from the centroids,
// the named bfSolver feature in FP64, the separating-plane certificate at 1e-6); the lanes
// whose result is not certified then take the exact certified solver together.  The
// contact rule is bf()'s (bf.cpp:125) on the FP64 distance.
constexpr int kLearnedSweeps = 2;
constexpr double kLearnedRelTol = 1e-6;
__global__ void __launch_bounds__(128, 4) k_learned_survivors(delta_meshes m, const int32_t *__restrict__ pa,
                                                           const int32_t *__restrict__ pb, RawContacts rc,
                                                           DevStats *st) {
  dep_sync();
  __shared__ CertWarpSmem sm[4];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned long long cnt = *rc.sv_count;
  const int64_t n = (int64_t)cnt < rc.sv_cap ? (int64_t)cnt : rc.sv_cap;
  if (n == 0) return;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  unsigned exact = 0;
  for (int64_t base = ((int64_t)blockIdx.x * (blockDim.x >> 5) + warp) * 32; base < n; base += nwarps * 32) {
    const int64_t i = base + lane;
    const bool valid = i < n;
    const uint64_t key = rc.sv[valid ? i : n - 1];
    RowCtx r;
    r.k = (int64_t)(key >> 32);
    r.iA = (int32_t)((key >> 16) & 0xffff);
    const int32_t tb = (int32_t)(key & 0xffff);
    const int32_t a = pa[r.k], b = pb[r.k];
    r.tA = m.tri_offset[a] + r.iA;
    r.tB0 = m.tri_offset[b];
    r.epsA = m.eps[a];
    r.epsB = m.eps[b];
    r.idA = m.id[a];
    r.idB = m.id[b];
    r.fric = (m.friction[a] && m.friction[b]) ? 1 : 0;
    double A[3][3], B[3][3], pq[6];
    load_tri_cur(m, rc.pose, a, r.tA, A);
    load_tri_cur(m, rc.pose, b, r.tB0 + tb, B);
    const bool ok = learned_pair_solve(A, B, kLearnedSweeps, kLearnedRelTol, pq);
    const bool need = valid && !ok;
    if (__any_sync(kFull, need)) {
      double px[6];
      bf_cert_warp(A, B, need, px, sm[warp]);
      if (need) {
#pragma unroll
        for (int k = 0; k < 6; ++k) pq[k] = px[k];
      }
      exact += need ? 1u : 0u;
    }
    const double mg = (xf64(r.epsA) + xf64(r.epsB)).v;
    emit(rc, valid && pq_dist64(pq) <= mg, pq, r, tb);  // bf.cpp:125
  }
  const unsigned tot = __reduce_add_sync(kFull, exact);
  if (lane == 0 && tot) atomicAdd(&st->penalty_fails, (unsigned long long)tot);  // pairs solved exactly
}

// The survivors' solver of a culled driver: certified FP32 + FP64 (DELTA_DRV_BF_CERT), FP64
// bfSolver (DELTA_DRV_BF_CULLED) or the learned FP32 hybrid (DELTA_DRV_LEARNED).
inline cudaError_t launch_survivors(int driver, cudaStream_t s, const delta_meshes &m, const int32_t *pa,
                                    const int32_t *pb, const RawContacts &rc, DevStats *st, int64_t n_hint,
                                    int cap = 0, bool dep = false) {
  int per_sm = 0;
  cudaError_t e = driver == DELTA_DRV_BF_CULLED
                      ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bf64_survivors, 128, 0)
                  : driver == DELTA_DRV_LEARNED
                      ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_learned_survivors, 128, 0)
                      : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cert_survivors, 128, 0);
  if (e != cudaSuccess) return e;
  if (cap > 0 && cap < per_sm) per_sm = cap;
  int64_t blocks = n_hint >= 0 ? (n_hint + 127) / 128 : INT64_MAX;
  const int64_t mx = (int64_t)kNumSMs * (per_sm > 0 ? per_sm : 1);
  if (blocks > mx) blocks = mx;
  if (blocks < 1) blocks = 1;
  if (driver == DELTA_DRV_BF_CULLED) return launch_dep(dep, k_bf64_survivors, (unsigned)blocks, 128, 0, s, m, pa, pb, rc);
  if (driver == DELTA_DRV_LEARNED)
    return launch_dep(dep, k_learned_survivors, (unsigned)blocks, 128, 0, s, m, pa, pb, rc, st);
  return launch_dep(dep, k_cert_survivors, (unsigned)blocks, 128, 0, s, m, pa, pb, rc, st);
}

__global__ void k_sv_evaluated(const unsigned long long *sv_count, int64_t sv_cap, DevStats *st, int *ovf) {
  const unsigned long long c = *sv_count;
  st->evaluated += c;
  if (ovf && c > (unsigned long long)sv_cap) atomicCAS(ovf, 0, 1);
}

__global__ void k_rows_per_pair(const int64_t *tri_offset, const int32_t *pa, int64_t n_pairs, int32_t n_bodies,
                                int64_t *rows, int *bad) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_pairs) return;
  const int32_t a = pa[k];
  if (a < 0 || a >= n_bodies) {
    atomicExch(bad, 1);
    rows[k] = 0;
    return;
  }
  rows[k] = tri_offset[a + 1] - tri_offset[a];
}

__global__ void k_rows_fixed(const int64_t *tri_offset, const int32_t *pa, int64_t cap, int64_t *rows) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k > cap) return;
  if (k == cap) { rows[k] = 0; return; }
  const int32_t a = pa[k];
  rows[k] = a < 0 ? 0 : tri_offset[a + 1] - tri_offset[a];
}

// Gather for the fixed-capacity path: count and overflow live on the device.
__global__ void k_gather_fixed(RawContacts rc, const int64_t *perm, delta_contacts out, int64_t *n_out, int *ovf,
                               int ovf_code, int64_t *count_log) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned long long cnt = *rc.count;
  const int64_t n = (int64_t)cnt < out.capacity ? (int64_t)cnt : out.capacity;
  if (j == 0) {
    *n_out = n;
    if (count_log) *count_log = n;
    if ((int64_t)cnt > out.capacity) atomicCAS(ovf, 0, ovf_code);
  }
  if (j >= n) return;
  const int64_t s = perm[j], cap = rc.cap, oc = out.capacity;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    out.x[k * oc + j] = rc.f[(0 + k) * cap + s];
    out.normal[k * oc + j] = rc.f[(3 + k) * cap + s];
    out.P[k * oc + j] = rc.f[(7 + k) * cap + s];
    out.Q[k * oc + j] = rc.f[(10 + k) * cap + s];
  }
  out.depth[j] = rc.f[6 * cap + s];
  out.eps_total[j] = rc.f[13 * cap + s];
  out.master[j] = rc.i[s];
  out.slave[j] = rc.i[cap + s];
  out.tri_a[j] = rc.i[2 * cap + s];
  out.tri_b[j] = rc.i[3 * cap + s];
  out.penetration[j] = 1;
  out.friction[j] = rc.fric[s];
}

// Sort-free ordering of the fixed-capacity certified driver's contacts, step 1: contact c
// of pair k goes to its pair's bucket, at poff[k] + its rank of arrival, with its key.
__global__ void k_bucket_contacts(RawContacts rc, const int64_t *poff, int64_t *bidx, uint64_t *bkey) {
  dep_sync();
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned long long cnt = *rc.count;
  const int64_t n = (int64_t)cnt < rc.cap ? (int64_t)cnt : rc.cap;
  if (c >= n) return;
  const uint64_t key = rc.key[c];
  const int64_t j = poff[(int64_t)(key >> (2 * rc.tbits))] + rc.slot[c];
  bidx[j] = c;
  bkey[j] = key;
}

// Step 2, one thread per bucket entry j: its pair k is the last with poff[k] <= j, its
// rank the number of smaller keys in the pair's bucket (keys within a pair are distinct),
// and the contact is written at poff[k] + rank, so the output is in (pair, A triangle,
// B triangle) order, the order of a stable sort of all keys.  Thread 0 publishes the
// count and flags an overflow.
__global__ void k_pair_gather(RawContacts rc, const int64_t *poff, const int64_t *bidx, const uint64_t *bkey,
                              int64_t n_pairs, delta_contacts out, int64_t *n_out, int *ovf, int ovf_code,
                              int64_t *count_log) {
  dep_sync();
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned long long cnt = *rc.count;
  if (j == 0) {
    const int64_t n = (int64_t)cnt < out.capacity ? (int64_t)cnt : out.capacity;
    *n_out = n;
    if (count_log) *count_log = n;
    if ((int64_t)cnt > out.capacity) atomicCAS(ovf, 0, ovf_code);
  }
  if (j >= poff[n_pairs]) return;
  int64_t lo = 0, hi = n_pairs;  // poff[0] = 0 <= j < poff[n_pairs]
  while (lo < hi) {
    const int64_t mid = (lo + hi + 1) >> 1;
    if (poff[mid] <= j) lo = mid;
    else hi = mid - 1;
  }
  const int64_t base = poff[lo], m = poff[lo + 1] - base;
  const uint64_t key = bkey[j];
  int64_t rank = 0;
  for (int64_t i = 0; i < m; ++i) rank += bkey[base + i] < key ? 1 : 0;
  const int64_t d = base + rank, s = bidx[j], cap = rc.cap, oc = out.capacity;
  if (d >= oc) return;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    out.x[k * oc + d] = rc.f[(0 + k) * cap + s];
    out.normal[k * oc + d] = rc.f[(3 + k) * cap + s];
    out.P[k * oc + d] = rc.f[(7 + k) * cap + s];
    out.Q[k * oc + d] = rc.f[(10 + k) * cap + s];
  }
  out.depth[d] = rc.f[6 * cap + s];
  out.eps_total[d] = rc.f[13 * cap + s];
  out.master[d] = rc.i[s];
  out.slave[d] = rc.i[cap + s];
  out.tri_a[d] = rc.i[2 * cap + s];
  out.tri_b[d] = rc.i[3 * cap + s];
  out.penetration[d] = 1;
  out.friction[d] = rc.fric[s];
}

__global__ void k_accumulate(const DevStats *st, int64_t *counters) {
  counters[0] += (int64_t)st->tri_pairs;
  counters[1] += (int64_t)st->evaluated;
}

// End of a fixed-capacity certified detection, one thread: the survivors count as
// evaluated pairs (a survivor-list overflow raises *ovf), then the step's statistics go
// to the running counters.
__global__ void k_cert_tail(const unsigned long long *sv_count, int64_t sv_cap, DevStats *st, int *ovf,
                            int64_t *counters, unsigned long long *queue) {
  dep_sync();
  const unsigned long long c = *sv_count;
  st->evaluated += c;
  if (ovf && c > (unsigned long long)sv_cap) atomicCAS(ovf, 0, 1);
  if (counters) {
    counters[0] += (int64_t)st->tri_pairs;
    counters[1] += (int64_t)st->evaluated;
  }
  if (queue) {  // fixed-capacity state: cleared for the next step (the step's last reader)
    queue[0] = queue[1] = queue[2] = 0ull;
    *st = DevStats{};
  }
}

__global__ void k_check_pairs(const int64_t *tri_offset, const int32_t *pb, int64_t n_pairs, int32_t n_bodies,
                              int *bad) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_pairs) return;
  const int32_t b = pb[k];
  if (b < 0 || b >= n_bodies) atomicExch(bad, 1);
}

__global__ void k_max_tris(const int64_t *tri_offset, int32_t n_bodies, int *bad) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_bodies) return;
  const int64_t n = tri_offset[i + 1] - tri_offset[i];
  if (n < 0 || n >= 65536) atomicExch(bad, 2);
}

__global__ void k_iota(int64_t *v, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = i;
}

__global__ void k_gather(RawContacts rc, const int64_t *perm, int64_t n, delta_contacts out) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int64_t s = perm[j], cap = rc.cap, oc = out.capacity;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    out.x[k * oc + j] = rc.f[(0 + k) * cap + s];
    out.normal[k * oc + j] = rc.f[(3 + k) * cap + s];
    out.P[k * oc + j] = rc.f[(7 + k) * cap + s];
    out.Q[k * oc + j] = rc.f[(10 + k) * cap + s];
  }
  out.depth[j] = rc.f[6 * cap + s];
  out.eps_total[j] = rc.f[13 * cap + s];
  out.master[j] = rc.i[s];
  out.slave[j] = rc.i[cap + s];
  out.tri_a[j] = rc.i[2 * cap + s];
  out.tri_b[j] = rc.i[3 * cap + s];
  out.penetration[j] = 1;
  out.friction[j] = rc.fric[s];
}

template <class R, int DRV>
cudaError_t launch_detect_t(cudaStream_t s, const delta_meshes &m, const int32_t *pa, const int32_t *pb,
                            const int64_t *row_offset, int64_t n_pairs, int64_t rows_hint, const RawContacts &rc,
                            DevStats *st, unsigned long long *queue) {
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_detect<R, DRV>, 128, 0);
  if (e != cudaSuccess) return e;
  int64_t blocks = (int64_t)kNumSMs * (per_sm > 0 ? per_sm : 1);
  if (rows_hint >= 0) {
    const int64_t need = (rows_hint + 3) / 4;  // 4 warps per block
    if (blocks > need) blocks = need > 0 ? need : 1;
  }
  k_detect<R, DRV><<<(unsigned)blocks, 128, 0, s>>>(m, pa, pb, row_offset, n_pairs, row_offset + n_pairs, rc, st,
                                                    queue);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_detect_prec(int driver, cudaStream_t s, const delta_meshes &m, const int32_t *pa,
                               const int32_t *pb, const int64_t *ro, int64_t np, int64_t rows,
                               const RawContacts &rc, DevStats *st, unsigned long long *q) {
  switch (driver) {
    case DELTA_DRV_BF: return launch_detect_t<R, DELTA_DRV_BF>(s, m, pa, pb, ro, np, rows, rc, st, q);
    case DELTA_DRV_PENALTY: return launch_detect_t<R, DELTA_DRV_PENALTY>(s, m, pa, pb, ro, np, rows, rc, st, q);
    case DELTA_DRV_PENALTY_STAT:
      return launch_detect_t<R, DELTA_DRV_PENALTY_STAT>(s, m, pa, pb, ro, np, rows, rc, st, q);
    case DELTA_DRV_HYBRID_BATCH:
      return launch_detect_t<R, DELTA_DRV_HYBRID_BATCH>(s, m, pa, pb, ro, np, rows, rc, st, q);
    case DELTA_DRV_HYBRID_TRIANGLE:
      return launch_detect_t<R, DELTA_DRV_HYBRID_TRIANGLE>(s, m, pa, pb, ro, np, rows, rc, st, q);
    case DELTA_DRV_HYBRID_BATCH_STAT:
      return launch_detect_t<R, DELTA_DRV_HYBRID_BATCH_STAT>(s, m, pa, pb, ro, np, rows, rc, st, q);
    case DELTA_DRV_HYBRID_TRI_STAT:
      return launch_detect_t<R, DELTA_DRV_HYBRID_TRI_STAT>(s, m, pa, pb, ro, np, rows, rc, st, q);
    case DELTA_DRV_GJK: return launch_detect_t<R, DELTA_DRV_GJK>(s, m, pa, pb, ro, np, rows, rc, st, q);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

cudaError_t detect_launch_limits(int driver, int *cull_per_sm, int *surv_per_sm) {
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(cull_per_sm, k_cull_pairs, kCullThreads, 0);
  if (e != cudaSuccess) return e;
  return driver == DELTA_DRV_BF_CULLED
             ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(surv_per_sm, k_bf64_survivors, 128, 0)
         : driver == DELTA_DRV_LEARNED
             ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(surv_per_sm, k_learned_survivors, 128, 0)
             : cudaOccupancyMaxActiveBlocksPerMultiprocessor(surv_per_sm, k_cert_survivors, 128, 0);
}

// Scratch slots used here: 2 rows/row_offset, 3 raw contacts, 4 sort buffers, 5 small state.
delta_status detect_run(delta_ctx *ctx, int driver, int precision, const delta_meshes &m, const int32_t *pa,
                        const int32_t *pb, int64_t n_pairs, const delta_contacts *out, int64_t *n_out,
                        delta_stats *stats, int64_t *counters, const Pose *pose) {
  cudaStream_t s = ctx->stream;
  delta_status st;
  cudaError_t e;
  // small device state: [0] bad flag (int), then DevStats, queue counter, contact counter
  void *small = nullptr;
  const size_t small_bytes = 256 + sizeof(DevStats) + 64;
  if ((st = ctx_scratch(ctx, 5, small_bytes, &small)) != DELTA_OK) return st;
  int *bad = (int *)small;
  DevStats *dstats = (DevStats *)((char *)small + 256);
  unsigned long long *queue = (unsigned long long *)((char *)small + 256 + sizeof(DevStats));
  unsigned long long *count = queue + 1;
  unsigned long long *sv_count = queue + 2;
  if ((e = cudaMemsetAsync(small, 0, small_bytes, s)) != cudaSuccess) return cuda_error(e, "detect memset");

  // rows per pair and their exclusive prefix sum
  void *rbuf = nullptr;
  if ((st = ctx_scratch(ctx, 2, sizeof(int64_t) * (size_t)(2 * n_pairs + 2), &rbuf)) != DELTA_OK) return st;
  int64_t *rows = (int64_t *)rbuf, *row_offset = rows + n_pairs + 1;
  const unsigned g = (unsigned)((n_pairs + 255) / 256);
  k_rows_per_pair<<<g, 256, 0, s>>>(m.tri_offset, pa, n_pairs, m.n_bodies, rows, bad);
  k_check_pairs<<<g, 256, 0, s>>>(m.tri_offset, pb, n_pairs, m.n_bodies, bad);
  k_max_tris<<<(unsigned)((m.n_bodies + 255) / 256), 256, 0, s>>>(m.tri_offset, m.n_bodies, bad);
  ctx->launches += 3;
  if ((e = cudaMemsetAsync(rows + n_pairs, 0, sizeof(int64_t), s)) != cudaSuccess) return cuda_error(e, "memset");
  size_t temp_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, temp_bytes, rows, row_offset, n_pairs + 1, s);
  void *temp = nullptr;
  if ((st = ctx_scratch(ctx, 4, temp_bytes, &temp)) != DELTA_OK) return st;
  if ((e = cub::DeviceScan::ExclusiveSum(temp, temp_bytes, rows, row_offset, n_pairs + 1, s)) != cudaSuccess)
    return cuda_error(e, "row scan");
  ctx->launches += 1;
  int64_t total_rows = 0;
  int hbad = 0;
  if ((e = cudaMemcpyAsync(&total_rows, row_offset + n_pairs, sizeof(int64_t), cudaMemcpyDeviceToHost, s)) !=
          cudaSuccess ||
      (e = cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return cuda_error(e, "detect rows");
  if (hbad == 1) return set_error(DELTA_ERR_INVALID, "delta_detect: body index out of range");
  if (hbad == 2) return set_error(DELTA_ERR_INVALID, "delta_detect: a body has 65536 or more triangles");

  // raw contact buffer: at least the caller's capacity; grown and rerun when it overflows
  int64_t cap = out->capacity > 1024 ? out->capacity : 1024;
  unsigned long long hcount = 0;
  RawContacts rc{};
  rc.tbits = 16;
  const bool culled = driver == DELTA_DRV_BF_CERT || driver == DELTA_DRV_BF_CULLED || driver == DELTA_DRV_LEARNED;
  if (culled && !cull_stride()) rc.pair_queue = queue;  // zeroed below before every culling launch
  if (culled && pose) {
    rc.pose = *pose;  // current vertices and body boxes from the bodies' poses
  } else if (culled) {
    // body boxes of the current vertices for the culling
    void *bb = nullptr;
    if ((st = ctx_scratch(ctx, 23, 48 * (size_t)m.n_bodies + 64, &bb)) != DELTA_OK) return st;
    const int64_t warps = std::min<int64_t>(m.n_bodies, (int64_t)kNumSMs * 64);
    k_body_boxes<<<(unsigned)std::max<int64_t>(1, (warps * 32 + 127) / 128), 128, 0, s>>>(m, (double *)bb);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(e, "body boxes");
    ctx->launches += 1;
    rc.bbox = (const double *)bb;
  }
  for (int attempt = 0; attempt < 2; ++attempt) {
    void *raw = nullptr;
    const size_t per = 14 * sizeof(double) + 4 * sizeof(int32_t) + 1 + 2 * sizeof(uint64_t);
    if ((st = ctx_scratch(ctx, 3, per * (size_t)cap + 64, &raw)) != DELTA_OK) return st;
    rc.cap = cap;
    rc.f = (double *)raw;
    rc.key = (uint64_t *)(rc.f + 14 * cap);
    rc.i = (int32_t *)(rc.key + 2 * cap);
    rc.fric = (uint8_t *)(rc.i + 4 * cap);
    rc.count = count;
    rc.sv_count = sv_count;
    if ((e = cudaMemsetAsync(queue, 0, 3 * sizeof(unsigned long long), s)) != cudaSuccess)
      return cuda_error(e, "memset");
    if ((e = cudaMemsetAsync(dstats, 0, sizeof(DevStats), s)) != cudaSuccess) return cuda_error(e, "memset");
    if (culled) {
      // phase 1: box culling into the survivor list (grown and repeated on overflow);
      // phase 2: the survivors' solver (certified bf, full warps across pairs; or FP64 bf)
      int64_t sv_cap = 8 * cap > (1 << 16) ? 8 * cap : (1 << 16);
      unsigned long long hsv = 0;
      for (int sv_attempt = 0; sv_attempt < 2; ++sv_attempt) {
        void *svb = nullptr;
        if ((st = ctx_scratch(ctx, 9, sizeof(uint64_t) * (size_t)sv_cap, &svb)) != DELTA_OK) return st;
        rc.sv = (uint64_t *)svb;
        rc.sv_cap = sv_cap;
        if ((e = cudaMemsetAsync(queue, 0, 3 * sizeof(unsigned long long), s)) != cudaSuccess)
          return cuda_error(e, "memset");
        if ((e = launch_cull(s, m, pa, pb, n_pairs, rc, dstats, ctx->cull_blocks_per_sm)) != cudaSuccess)
          return cuda_error(e, "cull kernel");
        ctx->launches += 1;
        if ((e = cudaMemcpyAsync(&hsv, sv_count, sizeof(hsv), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess)
          return cuda_error(e, "survivor count");
        if ((int64_t)hsv <= sv_cap) break;
        sv_cap = (int64_t)hsv + hsv / 4;
      }
      if ((e = launch_survivors(driver, s, m, pa, pb, rc, dstats, (int64_t)hsv, ctx->surv_blocks_per_sm)) !=
          cudaSuccess)
        return cuda_error(e, "survivor kernel");
      k_sv_evaluated<<<1, 1, 0, s>>>(sv_count, rc.sv_cap, dstats, nullptr);
      ctx->launches += 2;
      e = cudaGetLastError();
    } else {
      e = precision == DELTA_F32
            ? launch_detect_prec<float>(driver, s, m, pa, pb, row_offset, n_pairs, total_rows, rc, dstats, queue)
            : launch_detect_prec<xf64>(driver, s, m, pa, pb, row_offset, n_pairs, total_rows, rc, dstats, queue);
      ctx->launches += 1;
    }
    if (e != cudaSuccess) return cuda_error(e, "detect kernel");
    if ((e = cudaMemcpyAsync(&hcount, count, sizeof(hcount), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
      return cuda_error(e, "detect count");
    if ((int64_t)hcount <= cap) break;
    cap = (int64_t)hcount + hcount / 4;
  }
  if (stats || counters) {
    DevStats h;
    if ((e = cudaMemcpy(&h, dstats, sizeof h, cudaMemcpyDeviceToHost)) != cudaSuccess)
      return cuda_error(e, "stats");
    if (counters) {
      counters[0] += (int64_t)h.tri_pairs;
      counters[1] += (int64_t)h.evaluated;
    }
  }
  if (stats) {
    DevStats h;
    if ((e = cudaMemcpy(&h, dstats, sizeof h, cudaMemcpyDeviceToHost)) != cudaSuccess)
      return cuda_error(e, "stats");
    for (int i = 0; i < 17; ++i) stats->newton_hist[i] = (int64_t)h.hist[i];
    stats->penalty_fails = (int64_t)h.penalty_fails;
    stats->batch_fails = (int64_t)h.batch_fails;
    stats->batch_size = (int64_t)h.batch_size;
    stats->batch_error = h.batch_error;
  }
  const int64_t n = (int64_t)hcount;
  *n_out = n;
  if (n == 0) return DELTA_OK;
  // sort (key, index) and gather into the caller's arrays
  int64_t *perm_in = nullptr;
  void *sbuf = nullptr;
  if ((st = ctx_scratch(ctx, 6, sizeof(int64_t) * 2 * (size_t)n + sizeof(uint64_t) * (size_t)n, &sbuf)) != DELTA_OK)
    return st;
  perm_in = (int64_t *)sbuf;
  int64_t *perm_out = perm_in + n;
  uint64_t *key_out = (uint64_t *)(perm_out + n);
  k_iota<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(perm_in, n);
  ctx->launches += 1;
  int end_bit = 33;
  while (end_bit < 64 && ((int64_t)1 << (end_bit - 32)) < n_pairs) ++end_bit;
  temp_bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, rc.key, key_out, perm_in, perm_out, n, 0, end_bit, s);
  if ((st = ctx_scratch(ctx, 4, temp_bytes, &temp)) != DELTA_OK) return st;
  if ((e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, rc.key, key_out, perm_in, perm_out, n, 0, end_bit, s)) !=
      cudaSuccess)
    return cuda_error(e, "contact sort");
  ctx->launches += 1;
  const int64_t wn = n < out->capacity ? n : out->capacity;
  if (wn > 0) {
    k_gather<<<(unsigned)((wn + 255) / 256), 256, 0, s>>>(rc, perm_out, wn, *out);
    ctx->launches += 1;
  }
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_error(e, "detect gather");
  if (n > out->capacity) return set_error(DELTA_ERR_CAPACITY, "delta_detect: contact capacity exceeded");
  return DELTA_OK;
}

// Fixed-capacity detection for graph capture: pair_cap pairs (entries with a negative
// body index are empty), raw contact buffer and output of out->capacity entries, counts
// and overflow on the device.  Scratch (slots 13, 14) must have been sized by
// detect_fixed_prepare before capture.
size_t detect_fixed_temp_bytes(int64_t pair_cap, int64_t cap) {
  size_t a = 0, b = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, a, (int64_t *)nullptr, (int64_t *)nullptr, pair_cap + 1);
  cub::DeviceRadixSort::SortPairs(nullptr, b, (uint64_t *)nullptr, (uint64_t *)nullptr, (int64_t *)nullptr,
                                  (int64_t *)nullptr, cap, 0, 64);
  return a > b ? a : b;
}

static int64_t fixed_sv_cap(int64_t cap) { return 32 * cap > (1 << 16) ? 32 * cap : (1 << 16); }

size_t detect_fixed_state_bytes(int64_t pair_cap, int64_t cap) {
  const size_t per = 14 * sizeof(double) + 4 * sizeof(int32_t) + 1 + 2 * sizeof(uint64_t);
  return 512 + sizeof(DevStats) + sizeof(int64_t) * (size_t)(2 * pair_cap + 2) + per * (size_t)cap +
         sizeof(int64_t) * 2 * (size_t)cap + 256 + sizeof(uint64_t) * (size_t)fixed_sv_cap(cap) + 256;
}

// Once per allocation of the fixed-capacity state: the contact sort's identity permutation.
delta_status detect_fixed_init(cudaStream_t s, void *state, int64_t pair_cap, int64_t cap) {
  // the queue, counts and statistics start at zero; the culled drivers' tail kernel clears
  // them after each step, the other drivers' steps before
  cudaError_t e = cudaMemsetAsync(state, 0, 512 + sizeof(DevStats), s);
  if (e != cudaSuccess) return cuda_error(e, "detect fixed init");
  char *p = (char *)state + 512 + sizeof(DevStats) + sizeof(int64_t) * (size_t)(2 * pair_cap + 2);
  p += (14 * sizeof(double) + 4 * sizeof(int32_t) + 1 + 2 * sizeof(uint64_t)) * (size_t)cap;
  p = (char *)(((uintptr_t)p + 255) & ~(uintptr_t)255);
  k_iota<<<(unsigned)((cap + 255) / 256), 256, 0, s>>>((int64_t *)p, cap);
  return cuda_error(cudaGetLastError(), "detect fixed init");
}

delta_status detect_run_fixed(delta_ctx *ctx, cudaStream_t s, int driver, const delta_meshes &m, const int32_t *pa,
                              const int32_t *pb, int64_t pair_cap, const delta_contacts &out, int64_t *d_ncontacts,
                              int *d_ovf, int ovf_code, int64_t *d_counters, int64_t *d_count_log, void *state,
                              void *temp, size_t temp_bytes, const Pose *pose, int tri_bits) {
  cudaError_t e;
  const int64_t cap = out.capacity;
  char *p = (char *)state;
  unsigned long long *queue = (unsigned long long *)p;  // [0] queue [1] contact count
  DevStats *dstats = (DevStats *)(p + 256);
  p += 512 + sizeof(DevStats);
  int64_t *rows = (int64_t *)p, *row_offset = rows + pair_cap + 1;
  p += sizeof(int64_t) * (size_t)(2 * pair_cap + 2);
  RawContacts rc{};
  rc.tbits = tri_bits;
  rc.cap = cap;
  rc.f = (double *)p;
  rc.key = (uint64_t *)(rc.f + 14 * cap);
  rc.i = (int32_t *)(rc.key + 2 * cap);
  rc.fric = (uint8_t *)(rc.i + 4 * cap);
  rc.count = queue + 1;
  p += (14 * sizeof(double) + 4 * sizeof(int32_t) + 1 + 2 * sizeof(uint64_t)) * (size_t)cap;
  p = (char *)(((uintptr_t)p + 255) & ~(uintptr_t)255);
  int64_t *perm_in = (int64_t *)p, *perm_out = perm_in + cap;
  uint64_t *key_out = rc.key + cap;
  p += sizeof(int64_t) * 2 * (size_t)cap;
  p = (char *)(((uintptr_t)p + 255) & ~(uintptr_t)255);
  rc.sv = (uint64_t *)p;
  rc.sv_cap = fixed_sv_cap(cap);
  rc.sv_count = queue + 2;
  const bool culled = driver == DELTA_DRV_BF_CERT || driver == DELTA_DRV_BF_CULLED || driver == DELTA_DRV_LEARNED;
  if (culled && pose) rc.pose = *pose;  // vertices and body boxes from the poses
  if (culled && !cull_stride()) rc.pair_queue = queue;  // queue[0], zeroed with the state below
  // the culled drivers find the queue, counts and statistics cleared by the previous step's
  // tail kernel (or at allocation), so the culling follows the broadphase's last kernel
  // directly; the other drivers clear them here
  if (!culled && (e = cudaMemsetAsync(state, 0, 512 + sizeof(DevStats), s)) != cudaSuccess)
    return cuda_error(e, "memset");
  size_t tb = temp_bytes;
  if (culled) {
    // The culling takes body pairs directly (no rows).  The contacts are ordered without a
    // sort: counted per pair (rows, zeroed by the culling), the counts scanned into pair
    // offsets (row_offset), each contact put in its pair's bucket (indices in perm_out,
    // keys in perm_in, whose identity permutation serves only the other driver), and each
    // pair's bucket ranked by key.  The per-pair arrival ranks use the sort's key_out.
    rc.pcnt = (unsigned long long *)rows;
    rc.slot = (uint32_t *)key_out;
    // programmatic dependent launches (pdl.cuh)
    e = launch_cull(s, m, pa, pb, pair_cap, rc, dstats, ctx->cull_blocks_per_sm, true);
    if (e != cudaSuccess) return cuda_error(e, "cull kernel");
    if ((e = launch_survivors(driver, s, m, pa, pb, rc, dstats, -1, ctx->surv_blocks_per_sm, true)) != cudaSuccess)
      return cuda_error(e, "survivor kernel");
    if ((e = exclusive_sum(temp, tb, rows, row_offset, pair_cap + 1, s, true)) != cudaSuccess)
      return cuda_error(e, "pair contact scan");
    const unsigned cb = (unsigned)((cap + 255) / 256);
    if ((e = launch_dep(true, k_bucket_contacts, cb, 256, 0, s, rc, row_offset, perm_out, (uint64_t *)perm_in)) !=
            cudaSuccess ||
        (e = launch_dep(true, k_pair_gather, cb, 256, 0, s, rc, row_offset, perm_out, (const uint64_t *)perm_in,
                        pair_cap, out, d_ncontacts, d_ovf, ovf_code, d_count_log)) != cudaSuccess ||
        (e = launch_dep(true, k_cert_tail, 1, 1, 0, s, rc.sv_count, rc.sv_cap, dstats, d_ovf, d_counters, queue)) !=
            cudaSuccess)
      return cuda_error(e, "detect fixed");
    ctx->launches += 6;
    return DELTA_OK;
  } else {
    // empty key entries sort last
    if ((e = cudaMemsetAsync(rc.key, 0xff, sizeof(uint64_t) * cap, s)) != cudaSuccess) return cuda_error(e, "memset");
    k_rows_fixed<<<(unsigned)((pair_cap + 256) / 256), 256, 0, s>>>(m.tri_offset, pa, pair_cap, rows);
    if ((e = cub::DeviceScan::ExclusiveSum(temp, tb, rows, row_offset, pair_cap + 1, s)) != cudaSuccess)
      return cuda_error(e, "row scan");
    e = launch_detect_t<xf64, DELTA_DRV_BF>(s, m, pa, pb, row_offset, pair_cap, -1, rc, dstats, queue);
    ctx->launches += 3;
  }
  if (e != cudaSuccess) return cuda_error(e, "detect kernel");
  // perm_in holds 0 .. cap-1 from detect_fixed_init (the sort does not modify its inputs)
  // keys (pair << 2 tri_bits | A tri << tri_bits | B tri) of pairs below pair_cap: the bits
  // above the pair index are zero (empty entries, ~0, still sort last: stable, and after
  // every valid key)
  int end_bit = 2 * rc.tbits + 1;
  while (end_bit < 64 && ((int64_t)1 << (end_bit - 2 * rc.tbits)) < pair_cap) ++end_bit;
  tb = temp_bytes;
  if ((e = cub::DeviceRadixSort::SortPairs(temp, tb, rc.key, key_out, perm_in, perm_out, cap, 0, end_bit, s)) !=
      cudaSuccess)
    return cuda_error(e, "contact sort");
  k_gather_fixed<<<(unsigned)((cap + 255) / 256), 256, 0, s>>>(rc, perm_out, out, d_ncontacts, d_ovf, ovf_code,
                                                               d_count_log);
  ctx->launches += 2;
  if (d_counters) {
    k_accumulate<<<1, 1, 0, s>>>(dstats, d_counters);
    ctx->launches += 1;
  }
  return cuda_error(cudaGetLastError(), "detect fixed");
}

}  // namespace delta
