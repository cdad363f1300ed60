// step.cu -- forces, integration, broadphase and the time-step loop.
//
// All physics arithmetic is FP64 written over xf64, i.e. the rounded operations of the
// reference (forces.cpp, dynamics.cpp, MoveParticles.cpp) in their order, without FMA
// contraction.  Summations that the reference performs sequentially (contacts of one
// partner, then partners of one body) are kept sequential per pair / per body; no
// floating-point atomics are used, so results do not depend on scheduling.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pdl.cuh"
#include "blockscan.cuh"
#include "internal.h"
#include "pose.cuh"
#include "real.cuh"

namespace delta {

namespace {

using X = xf64;

// ---------------------------------------------------------------------------------------
// dynamics.cpp
// ---------------------------------------------------------------------------------------

struct BodyRef {
  int32_t n, i;
  __device__ __forceinline__ int64_t at(int c) const { return (int64_t)c * n + i; }
};

// updateRotationMatrix, dynamics.cpp:104-138
__device__ __forceinline__ void update_rotation(const delta_scene &s, BodyRef b, X step) {
  X W[3], R0[9], DL[9];
#pragma unroll
  for (int k = 0; k < 3; ++k) W[k] = X(s.ref_ang[b.at(k)]);
#pragma unroll
  for (int k = 0; k < 9; ++k) R0[k] = X(s.rot[b.at(k)]);
  expmap(step * W[0], step * W[1], step * W[2], DL);
  X R[9];
#pragma unroll
  for (int col = 0; col < 3; ++col)
#pragma unroll
    for (int row = 0; row < 3; ++row)
      R[3 * col + row] = R0[row] * DL[3 * col] + R0[3 + row] * DL[3 * col + 1] + R0[6 + row] * DL[3 * col + 2];
#pragma unroll
  for (int k = 0; k < 9; ++k) s.rot[b.at(k)] = R[k].v;
#pragma unroll
  for (int row = 0; row < 3; ++row) s.ang[b.at(row)] = (R[row] * W[0] + R[3 + row] * W[1] + R[6 + row] * W[2]).v;
}

// updateAngular, dynamics.cpp:140-213 (eqs. 13-15)
__device__ __forceinline__ void update_angular(const delta_scene &s, BodyRef b, const X tq[3], X step) {
  X W[3], R[9], J[9], Ji[9];
#pragma unroll
  for (int k = 0; k < 3; ++k) W[k] = X(s.ref_ang[b.at(k)]);
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    R[k] = X(s.rot[b.at(k)]);
    J[k] = X(s.inertia[b.at(k)]);
    Ji[k] = X(s.inverse[b.at(k)]);
  }
  const X half = X(0.5) * step;
  X T[3], DL[9], A[3], B[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) T[i] = R[3 * i] * tq[0] + R[3 * i + 1] * tq[1] + R[3 * i + 2] * tq[2];
  expmap(-half * W[0], -half * W[1], -half * W[2], DL);
#pragma unroll
  for (int i = 0; i < 3; ++i) A[i] = J[i] * W[0] + J[3 + i] * W[1] + J[6 + i] * W[2];
#pragma unroll
  for (int i = 0; i < 3; ++i) B[i] = DL[i] * A[0] + DL[3 + i] * A[1] + DL[6 + i] * A[2];
#pragma unroll
  for (int i = 0; i < 3; ++i) B[i] = B[i] + half * T[i];
#pragma unroll
  for (int i = 0; i < 3; ++i) A[i] = Ji[i] * B[0] + Ji[3 + i] * B[1] + Ji[6 + i] * B[2];
#pragma unroll
  for (int i = 0; i < 3; ++i) B[i] = J[i] * A[0] + J[3 + i] * A[1] + J[6 + i] * A[2];
  T[0] -= A[1] * B[2] - A[2] * B[1];
  T[1] -= A[2] * B[0] - A[0] * B[2];
  T[2] -= A[0] * B[1] - A[1] * B[0];
  T[0] *= step;
  T[1] *= step;
  T[2] *= step;
#pragma unroll
  for (int i = 0; i < 3; ++i) s.ref_ang[b.at(i)] = (W[i] + Ji[i] * T[0] + Ji[3 + i] * T[1] + Ji[6 + i] * T[2]).v;
}

// ---------------------------------------------------------------------------------------
// forces.cpp
// ---------------------------------------------------------------------------------------

struct ContactView {
  const double *x, *normal, *depth;
  const int32_t *master, *slave;
  const uint8_t *friction;
  int64_t cap;
};

// State of one body as the contact forces read it.
struct BodyKin {
  X pos[3], ang[3], lin[3], mass;
};

__device__ __forceinline__ BodyKin body_kin(const delta_scene &s, int32_t a) {
  const int32_t n = s.n_bodies;
  BodyKin k;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    k.pos[d] = X(s.pos[(int64_t)d * n + a]);
    k.ang[d] = X(s.ang[(int64_t)d * n + a]);
    k.lin[d] = X(s.vel[(int64_t)d * n + a]);
  }
  k.mass = X(s.mass[a]);
  return k;
}

// The terms of one contact c in getContactsForces (forces.cpp:23-396): the force term
// (spring + damping + friction) and the torque term that the loop adds to its sums, for
// body A against B; `negate` applies the inverted normal stored for the slave
// (Collision.cpp:176-184).  Each term is formed in full before it is added, so a sum of
// these terms in list order is the reference loop's sum bit for bit.
__device__ __forceinline__ void contact_terms(const ContactView &cv, int64_t c, const BodyKin &A, const BodyKin &B,
                                              bool negate, const delta_step_params &p, X Fc[3], X Tc[3]) {
  const X spring = X(p.spring), damper = X(p.damper), mu = X(p.friction);
  X x[3], nn[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    x[k] = X(cv.x[k * cv.cap + c]);
    const X nv = X(cv.normal[k * cv.cap + c]);
    nn[k] = negate ? X(-1.0) * nv : nv;
  }
  const X depth = X(cv.depth[c]);
  X z[3], vi[3], vj[3], vij[3];
  for (int k = 0; k < 3; ++k) z[k] = x[k] - A.pos[k];
  vi[0] = A.ang[1] * z[2] - A.ang[2] * z[1] + A.lin[0];
  vi[1] = A.ang[2] * z[0] - A.ang[0] * z[2] + A.lin[1];
  vi[2] = A.ang[0] * z[1] - A.ang[1] * z[0] + A.lin[2];
  for (int k = 0; k < 3; ++k) z[k] = x[k] - B.pos[k];
  vj[0] = B.ang[1] * z[2] - B.ang[2] * z[1] + B.lin[0];
  vj[1] = B.ang[2] * z[0] - B.ang[0] * z[2] + B.lin[1];
  vj[2] = B.ang[0] * z[1] - B.ang[1] * z[0] + B.lin[2];
  for (int k = 0; k < 3; ++k) vij[k] = vj[k] - vi[k];
  const X ma = X(1.0) / ((X(1.0) / A.mass) + (X(1.0) / B.mass));
  const X velocity = (vij[0] * nn[0]) + (vij[1] * nn[1]) + (vij[2] * nn[2]);
  const X damp = damper * X(2.0) * sqrt_(ma * spring) * velocity;
  const X fmag = spring * depth + damp;
  X f[3], fr[3] = {X(0.0), X(0.0), X(0.0)};
  for (int k = 0; k < 3; ++k) f[k] = fmag * nn[k];
  if (cv.friction[c]) {
    const X vn = (vi[0] * nn[0]) + (vi[1] * nn[1]) + (vi[2] * nn[2]);
    for (int k = 0; k < 3; ++k) {
      const X vt = vi[k] - nn[k] * vn;
      fr[k] = -vt * mu * fmag;
    }
  }
  for (int k = 0; k < 3; ++k) Fc[k] = f[k] + fr[k];
  X arm[3];
  for (int k = 0; k < 3; ++k) arm[k] = x[k] - A.pos[k];
  Tc[0] = arm[1] * (f[2]) - arm[2] * (f[1]);
  Tc[1] = arm[2] * (f[0]) - arm[0] * (f[2]);
  Tc[2] = arm[0] * (f[1]) - arm[1] * (f[0]);
}

// Last kernel of a graph step.  A step that integrated (no overflow before it) is counted
// and logged; its counters (pend: candidate pairs, triangle pairs, solved pairs, summed
// during the step) go to the running totals only if no overflow arose in it either: the
// host repeats an overflowing step's detection, with its counters, outside the graph, and
// the replays queued after it are frozen.  pend is cleared for the next step.
__global__ void k_step_end(const int *ovf_snap, const int *ovf, const int64_t *n_contacts, int64_t *log,
                           int64_t log_len, int64_t *step, int64_t *pend, int64_t *pairs_total, int64_t *counters) {
  dep_sync();
  if (!*ovf_snap) {
    const int64_t k = *step;
    if (k < log_len) log[k] = *n_contacts;
    *step = k + 1;
    if (!*ovf) {
      *pairs_total += pend[0];
      counters[0] += pend[1];
      counters[1] += pend[2];
    }
  }
  pend[0] = pend[1] = pend[2] = 0;
}

__global__ void k_segment_heads(ContactView cv, int64_t n, uint8_t *head) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  head[c] = (c == 0 || cv.master[c] != cv.master[c - 1] || cv.slave[c] != cv.slave[c - 1]) ? 1 : 0;
}

// Partner-pair force sums, one thread per contact.  Every thread forms its contact's terms
// for both sides (master: force and torque on the master; slave: with the inverted normal,
// on the slave) in shared memory.  The thread at the first contact of a (master, slave)
// segment then adds the segment's terms in contact order, forming itself the terms of
// contacts past its block.  From 0.0 in contact order, these are the sums of the
// getContactsForces loop over the pair's contacts (forces.cpp:23-396), bit for bit.
//  - kFixed (graph path, count on the device): the sums go to entry 2c (on the master) and
//    2c+1 (on the slave), c the segment's first contact, and the segment is counted in its
//    slave's list.  Sums on obstacles are not formed: nothing reads them.
//  - otherwise: segment g (seg_start[g] == c) gets entries 2g and 2g+1, keyed
//    (body << sh | partner) for the entry sort, sh the bits of a body index.
constexpr int kHeadThreads = 128;
template <bool kFixed>
__global__ void __launch_bounds__(kHeadThreads) k_pair_forces_heads(
    delta_scene s, ContactView cv, const int64_t *n_contacts_d, int64_t n_contacts_h, const int64_t *seg_start,
    const int64_t *n_seg_p, delta_step_params p, int sh, uint64_t *key, int64_t *val_idx, double *entry,
    uint32_t *slave_count) {
  dep_sync();
  __shared__ double term[12][kHeadThreads];  // master F, master T, slave F, slave T
  const int64_t blk0 = (int64_t)blockIdx.x * kHeadThreads;
  const int64_t c = blk0 + threadIdx.x;
  int64_t n = n_contacts_d ? *n_contacts_d : n_contacts_h;
  if (n > cv.cap) n = cv.cap;
  if (blk0 >= n) return;  // the whole block is past the contacts
  const int64_t blk1 = blk0 + kHeadThreads < n ? blk0 + kHeadThreads : n;
  int32_t i = 0, j = 0;
  bool oi = true, oj = true;
  if (c < n) {
    i = cv.master[c];
    j = cv.slave[c];
    oi = kFixed && s.obstacle[i] != 0;
    oj = kFixed && s.obstacle[j] != 0;
    const BodyKin Ki = body_kin(s, i), Kj = body_kin(s, j);
    X Fc[3], Tc[3];
    if (!oi) {
      contact_terms(cv, c, Ki, Kj, false, p, Fc, Tc);
      for (int k = 0; k < 3; ++k) {
        term[k][threadIdx.x] = Fc[k].v;
        term[3 + k][threadIdx.x] = Tc[k].v;
      }
    }
    if (!oj) {
      contact_terms(cv, c, Kj, Ki, true, p, Fc, Tc);
      for (int k = 0; k < 3; ++k) {
        term[6 + k][threadIdx.x] = Fc[k].v;
        term[9 + k][threadIdx.x] = Tc[k].v;
      }
    }
  }
  __syncthreads();
  if (c >= n) return;
  if (c > 0 && cv.master[c] == cv.master[c - 1] && cv.slave[c] == cv.slave[c - 1]) return;
  int64_t c1 = c + 1;
  while (c1 < n && cv.master[c1] == i && cv.slave[c1] == j) ++c1;
  int64_t e0 = 2 * c;
  if constexpr (!kFixed) {
    int64_t lo = 0, hi = *n_seg_p;  // the segment index: seg_start[g] == c
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (seg_start[mid] < c) lo = mid + 1;
      else hi = mid;
    }
    e0 = 2 * lo;
  }
  // the sums of one side: terms from shared memory within the block, formed here past it
  auto side = [&](int o, int32_t a, int32_t b, bool negate, int64_t e) {
    X F[3] = {X(0.0), X(0.0), X(0.0)}, T[3] = {X(0.0), X(0.0), X(0.0)};
    for (int64_t u = c; u < c1 && u < blk1; ++u) {
      const int t = (int)(u - blk0);
      for (int k = 0; k < 3; ++k) {
        F[k] += X(term[o + k][t]);
        T[k] += X(term[o + 3 + k][t]);
      }
    }
    if (c1 > blk1) {
      const BodyKin A = body_kin(s, a), B = body_kin(s, b);
      for (int64_t u = blk1; u < c1; ++u) {
        X Fc[3], Tc[3];
        contact_terms(cv, u, A, B, negate, p, Fc, Tc);
        for (int k = 0; k < 3; ++k) {
          F[k] += Fc[k];
          T[k] += Tc[k];
        }
      }
    }
    for (int k = 0; k < 3; ++k) {
      entry[e * 6 + k] = F[k].v;
      entry[e * 6 + 3 + k] = T[k].v;
    }
  };
  if (!oi) side(0, i, j, false, e0);
  if (!oj) side(6, j, i, true, e0 + 1);
  if constexpr (kFixed) {
    if (!oj) atomicAdd(&slave_count[j], 1u);
  } else {
    key[e0] = ((uint64_t)(uint32_t)i << sh) | (uint32_t)j;
    key[e0 + 1] = ((uint64_t)(uint32_t)j << sh) | (uint32_t)i;
    val_idx[e0] = e0;
    val_idx[e0 + 1] = e0 + 1;
  }
}

// Each segment head c into its slave's list, at any position of the slave's range (the
// sum kernel orders the range).
__global__ void k_fill_slave_lists(delta_scene s, ContactView cv, const int64_t *n_contacts_d, const uint32_t *start,
                                   uint32_t *fill, int32_t *list) {
  dep_sync();
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t n = *n_contacts_d < cv.cap ? *n_contacts_d : cv.cap;
  if (c >= n) return;
  if (c > 0 && cv.master[c] == cv.master[c - 1] && cv.slave[c] == cv.slave[c - 1]) return;
  const int32_t j = cv.slave[c];
  if (s.obstacle[j]) return;
  list[start[j] + atomicAdd(&fill[j], 1u)] = (int32_t)c;
}

// Per-body sums over ascending partners, one thread per body.  The pair list is ordered
// (min, max), so a body's partners below it are the masters of the segments in which it is
// the slave, and those above it the slaves of the segments in which it is the master.
// The first come from the body's list, sorted by segment position (which orders them by
// master); the second are the body's run of contacts as master, in contact order.  From
// 0.0, these are the additions of the sorted-entry sums (k_body_forces), in that order.
__global__ void k_body_forces_lists(delta_scene s, ContactView cv, const int64_t *n_contacts_d, const uint32_t *start,
                                    int32_t *list, const double *entry, double *force, double *torque, uint8_t *has,
                                    uint32_t *slave_count, uint32_t *fill) {
  dep_sync();
  const int32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  const int32_t nb = s.n_bodies;
  if (b >= nb) return;
  // the body's slave count and fill position, read by the kernels before this one, are
  // cleared for the next step (slave_count[nb] is never counted)
  slave_count[b] = 0u;
  fill[b] = 0u;
  X F[3] = {X(0.0), X(0.0), X(0.0)}, T[3] = {X(0.0), X(0.0), X(0.0)};
  bool any = false;
  auto add = [&](const double *v) {
    for (int k = 0; k < 3; ++k) {
      F[k] += X(v[k]);
      T[k] += X(v[3 + k]);
    }
    any = true;
  };
  if (!s.obstacle[b]) {
    const uint32_t l0 = start[b], l1 = start[b + 1];
    for (uint32_t u = l0 + 1; u < l1; ++u) {  // insertion sort of this body's short list
      const int32_t v = list[u];
      uint32_t w = u;
      while (w > l0 && list[w - 1] > v) {
        list[w] = list[w - 1];
        --w;
      }
      list[w] = v;
    }
    for (uint32_t u = l0; u < l1; ++u) add(entry + (2 * (int64_t)list[u] + 1) * 6);
    const int64_t n = *n_contacts_d < cv.cap ? *n_contacts_d : cv.cap;
    int64_t lo = 0, hi = n;  // first contact with master >= b (masters ascend)
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (cv.master[mid] < b) lo = mid + 1;
      else hi = mid;
    }
    for (int64_t c = lo; c < n && cv.master[c] == b; ++c)
      if (c == lo || cv.slave[c] != cv.slave[c - 1]) add(entry + (2 * c) * 6);
  }
  for (int k = 0; k < 3; ++k) {
    force[(int64_t)k * nb + b] = F[k].v;
    torque[(int64_t)k * nb + b] = T[k].v;
  }
  has[b] = any ? 1 : 0;
}

// Per-body sums over the sorted entries: the thread at the first entry of a body's run
// adds the run's entries in key order, i.e. over ascending partners, starting from 0.0.
// Bodies without entries keep the zeros written before the launch.  Entries past the
// valid ones carry the key ~0 and sort last.
__global__ void k_body_forces(int32_t n_bodies, int sh, const uint64_t *skey, const int64_t *sidx,
                              const double *entry, int64_t ne, double *force, double *torque, uint8_t *has) {
  const int64_t e0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e0 >= ne) return;
  const uint64_t key = skey[e0];
  if (key == ~0ull) return;
  const uint64_t body = key >> sh;
  if (e0 > 0 && (skey[e0 - 1] >> sh) == body) return;  // not the first entry of the run
  const int64_t i = (int64_t)body;
  X F[3] = {X(0.0), X(0.0), X(0.0)}, T[3] = {X(0.0), X(0.0), X(0.0)};
  // run end, then the run in groups of 4 entries whose loads are issued together (a body
  // such as a floor can have thousands of partners); the additions stay in entry order
  int64_t e1 = e0 + 1;
  while (e1 < ne && skey[e1] != ~0ull && (skey[e1] >> sh) == body) ++e1;
  for (int64_t e = e0; e < e1; e += 4) {
    double v[4][6];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (e + u < e1) {
        const double *src = entry + sidx[e + u] * 6;
#pragma unroll
        for (int k = 0; k < 6; ++k) v[u][k] = src[k];
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (e + u < e1) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          F[k] += X(v[u][k]);
          T[k] += X(v[u][3 + k]);
        }
      }
    }
  }
  for (int k = 0; k < 3; ++k) {
    force[(int64_t)k * n_bodies + i] = F[k].v;
    torque[(int64_t)k * n_bodies + i] = T[k].v;
  }
  has[i] = 1;
}

// zeroes the per-body sums (bodies without contacts keep these)
inline cudaError_t zero_body_sums(cudaStream_t st, int32_t n, double *force, double *torque, uint8_t *has) {
  if (torque == force + 3 * (size_t)n && has == reinterpret_cast<uint8_t *>(torque + 3 * (size_t)n))
    return cudaMemsetAsync(force, 0, sizeof(double) * 6 * (size_t)n + (size_t)n, st);  // one buffer
  cudaError_t e = cudaMemsetAsync(force, 0, sizeof(double) * 3 * (size_t)n, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(torque, 0, sizeof(double) * 3 * (size_t)n, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(has, 0, (size_t)n, st);
  return e;
}

// ---------------------------------------------------------------------------------------
// integration
// ---------------------------------------------------------------------------------------

// Collision::touchVertexFirstTime velocity part (Collision.cpp:1105-1115) followed by
// MoveParticles::moveAllParticlesAssociatedToVertex body part (MoveParticles.cpp:71-94).
// With ovf_snap (graph mode) the first thread also opens the step: it snapshots the
// overflow flag and advances the vertex-stamp epoch.
__global__ void k_bodies(delta_scene s, delta_step_params p, const double *force, const double *torque,
                         const uint8_t *has, const int *ovf, int *ovf_snap, uint32_t *epoch) {
  dep_sync();
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (ovf_snap && i == 0) {
    *ovf_snap = *ovf;
    *epoch += 1u;
  }
  if (i >= s.n_bodies || s.obstacle[i]) return;
  if (ovf && *ovf) return;  // graph mode: a capacity overflow froze the state
  const BodyRef b{s.n_bodies, i};
  const X dt = X(p.dt);
  if (has[i]) {
    const X m = X(s.mass[i]);
    X tq[3];
    for (int k = 0; k < 3; ++k) {
      s.vel[b.at(k)] = (X(s.vel[b.at(k)]) + dt * (X(force[b.at(k)]) / m)).v;
      tq[k] = X(torque[b.at(k)]);
    }
    update_angular(s, b, tq, dt);
  }
  for (int k = 0; k < 3; ++k) s.vel[b.at(k)] = (X(s.vel[b.at(k)]) + dt * (X(p.gravity[k]))).v;
  for (int k = 0; k < 3; ++k) s.pos[b.at(k)] = (X(s.pos[b.at(k)]) + dt * X(s.vel[b.at(k)])).v;
  update_rotation(s, b, dt);
}

// updateVertices, dynamics.cpp:215-242, one warp per body: the body's 15 scalars (R, pos,
// ref_pos) are loaded by lanes 0..14 and broadcast, the lanes then stride over the body's
// vertices.  With `bbox` given the kernel also writes the box (lo[3], hi[3]) of every body's
// current vertices, obstacles included, for the certified driver's culling.  With the
// overflow flag set no vertex moves (graph mode: the state is frozen) but the boxes are
// still written, so they always describe the vertices in memory.
// With `stamp`, only the bodies whose stamp equals *epoch (the bodies of this step's
// candidate pairs, k_mark_pair_bodies) are processed.
__global__ void k_vertices(delta_scene s, const int *ovf, double *bbox, const uint32_t *stamp, const uint32_t *epoch) {
  dep_sync();
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const bool frozen = ovf && *ovf;
  const uint32_t ep = stamp ? *epoch : 0u;
  const int32_t n = s.n_bodies;
  for (int64_t i = warp; i < n; i += nwarps) {
    if (stamp && stamp[i] != ep) continue;
    const bool move = !frozen && !s.obstacle[i];
    if (!move && !bbox) continue;
    double q = 0.0;
    if (move && lane < 15)
      q = lane < 9 ? s.rot[(int64_t)lane * n + i]
                   : (lane < 12 ? s.pos[(int64_t)(lane - 9) * n + i] : s.ref_pos[(int64_t)(lane - 12) * n + i]);
    X R[9], pos[3], rp[3];
#pragma unroll
    for (int k = 0; k < 9; ++k) R[k] = X(__shfl_sync(0xffffffffu, q, k));
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      pos[k] = X(__shfl_sync(0xffffffffu, q, 9 + k));
      rp[k] = X(__shfl_sync(0xffffffffu, q, 12 + k));
    }
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    const int64_t v1 = 3 * s.tri_offset[i + 1];
    // kU vertices per lane per pass, their loads issued together
    constexpr int kU = 4;
    for (int64_t base = 3 * s.tri_offset[i] + lane; base < v1; base += 32 * kU) {
      double c[kU][3];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int64_t v = base + 32 * u;
        if (v < v1) {
          c[u][0] = move ? s.rx[v] : s.x[v];
          c[u][1] = move ? s.ry[v] : s.y[v];
          c[u][2] = move ? s.rz[v] : s.z[v];
        }
      }
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int64_t v = base + 32 * u;
        if (v < v1) {
          if (move) {
            posed_point(R, pos, rp, c[u][0], c[u][1], c[u][2], c[u]);
            s.x[v] = c[u][0];
            s.y[v] = c[u][1];
            s.z[v] = c[u][2];
          }
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            lo[k] = fmin(lo[k], c[u][k]);
            hi[k] = fmax(hi[k], c[u][k]);
          }
        }
      }
    }
    if (bbox) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        for (int o = 16; o > 0; o >>= 1) {
          lo[k] = fmin(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
          hi[k] = fmax(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
        }
      }
      if (lane == 0)
        for (int k = 0; k < 3; ++k) {
          bbox[6 * i + k] = lo[k];
          bbox[6 * i + 3 + k] = hi[k];
        }
    }
  }
}

// bits of a value below 2^b with 2^b > v (at most 31): pair and force keys pack two body
// indices in 2*bits_for(n_bodies) bits so that their radix sorts take fewer passes
inline int bits_for(int64_t v) {
  int b = 1;
  while (b < 31 && ((int64_t)1 << b) <= v) ++b;
  return b;
}

// Next epoch of the vertex stamps (one thread).
__global__ void k_next_epoch(uint32_t *epoch) { *epoch += 1u; }

// Stamps both bodies of every pair (entries with a negative body are empty) with the
// current epoch: these are the bodies whose vertices the narrowphase reads this step.
__global__ void k_mark_pair_bodies(const int32_t *pa, const int32_t *pb, int64_t n, const uint32_t *epoch,
                                   uint32_t *stamp) {
  dep_sync();
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const uint32_t e = *epoch;
  const int32_t a = pa[t], b = pb[t];
  if (a >= 0) stamp[a] = e;
  if (b >= 0) stamp[b] = e;
}

// Once per simulation, one warp per body: a moving body's reach, the largest |r - ref_pos|
// over its reference vertices (each difference rounded as the vertex update rounds it),
// and an obstacle's box (lo[3], hi[3]) of its vertices, which never move.
__global__ void k_reach_boxes(delta_scene s, double *reach, double *obox) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int32_t n = s.n_bodies;
  for (int64_t i = warp; i < n; i += nwarps) {
    const bool obst = s.obstacle[i] != 0;
    double rp[3], r2 = 0.0, lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int k = 0; k < 3; ++k) rp[k] = s.ref_pos[(int64_t)k * n + i];
    for (int64_t v = 3 * s.tri_offset[i] + lane; v < 3 * s.tri_offset[i + 1]; v += 32) {
      if (obst) {
        const double c[3] = {s.x[v], s.y[v], s.z[v]};
        for (int k = 0; k < 3; ++k) {
          lo[k] = fmin(lo[k], c[k]);
          hi[k] = fmax(hi[k], c[k]);
        }
      } else {
        const double d0 = (X(s.rx[v]) - X(rp[0])).v, d1 = (X(s.ry[v]) - X(rp[1])).v, d2 = (X(s.rz[v]) - X(rp[2])).v;
        r2 = fmax(r2, d0 * d0 + d1 * d1 + d2 * d2);
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      r2 = fmax(r2, __shfl_xor_sync(0xffffffffu, r2, o));
      for (int k = 0; k < 3; ++k) {
        lo[k] = fmin(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
        hi[k] = fmax(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
      }
    }
    if (lane == 0) {
      reach[i] = sqrt(r2) * (1.0 + 1e-12);
      for (int k = 0; k < 3; ++k) {
        obox[6 * i + k] = lo[k];
        obox[6 * i + 3 + k] = hi[k];
      }
    }
  }
}

inline unsigned vertex_blocks(int32_t n_bodies) {
  const int64_t b = ((int64_t)n_bodies + 7) / 8;  // 8 warps per 256-thread block
  return (unsigned)(b < 1 ? 1 : (b > 8 * kNumSMs ? 8 * kNumSMs : b));
}

// ---------------------------------------------------------------------------------------
// broadphase: uniform grid for moving bodies, bounding boxes for obstacles
// ---------------------------------------------------------------------------------------

struct Grid {
  double h;
  double origin[3];
};

// The skin list's margin as a fraction of a grid cell (skin = cell / kSkinPerCell).
constexpr double kSkinPerCell = 32.0;

// Hash grid of the moving bodies.  A cell is keyed by its coordinates modulo 2^21
// (cells that far apart share a key; their bodies become extra candidates that
// spheres_touch rejects) and lives in bucket hash(key) & (nb - 1), nb a power of two.
// Buckets list their bodies in any order: the candidate pairs are sorted afterwards.
constexpr int kCellBits = 21;
constexpr int64_t kCellMask = (1 << kCellBits) - 1;

__device__ __forceinline__ uint64_t cell_key(int64_t cx, int64_t cy, int64_t cz) {
  return ((uint64_t)(cx & kCellMask) << (2 * kCellBits)) | ((uint64_t)(cy & kCellMask) << kCellBits) |
         (uint64_t)(cz & kCellMask);
}

__device__ __forceinline__ uint32_t cell_bucket(uint64_t key, int64_t nb) {
  uint64_t h = key * 0x9E3779B97F4A7C15ull;  // multiplicative hashing (Knuth), high bits
  return (uint32_t)(h >> 32) & (uint32_t)(nb - 1);
}

struct HashGrid {
  int64_t nb;        // buckets, a power of two
  uint32_t *count;   // [nb + 1], zero before the count pass (count[nb] stays 0)
  uint32_t *fill;    // [nb], zero before the fill pass
  uint32_t *start;   // [nb + 1], exclusive sum of count
  int32_t *bodies;   // [n] bodies by bucket
  uint64_t *cell;    // [n] cell key of each moving body
};

inline int64_t grid_buckets(int32_t n) {
  int64_t nb = 1024;
  while (nb < (int64_t)n) nb <<= 1;
  return nb;
}

__device__ __forceinline__ void cell_of(const delta_scene &s, const Grid &g, int32_t i, int64_t c[3]) {
#pragma unroll
  for (int k = 0; k < 3; ++k) c[k] = (int64_t)floor((s.pos[(int64_t)k * s.n_bodies + i] - g.origin[k]) / g.h);
}

// Count pass: each moving body's cell key and bucket count.  With `pk` (fixed
// capacity), the grid's threads also empty the pair-key list (pk_cap entries of ~0) and
// zero its counter before the pair search fills them.
__global__ void k_grid_count(delta_scene s, Grid g, HashGrid hg, uint64_t *pk, int64_t pk_cap,
                             unsigned long long *count) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (pk) {
    for (int64_t t = i; t < pk_cap; t += (int64_t)gridDim.x * blockDim.x) pk[t] = ~0ull;
    if (i == 0) *count = 0ull;
  }
  if (i >= s.n_bodies || s.obstacle[i]) return;
  int64_t c[3];
  cell_of(s, g, i, c);
  const uint64_t key = cell_key(c[0], c[1], c[2]);
  hg.cell[i] = key;
  atomicAdd(&hg.count[cell_bucket(key, hg.nb)], 1u);
}

// Fill pass: each moving body into its bucket.
__global__ void k_grid_fill(delta_scene s, HashGrid hg) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n_bodies || s.obstacle[i]) return;
  const uint32_t b = cell_bucket(hg.cell[i], hg.nb);
  hg.bodies[hg.start[b] + atomicAdd(&hg.fill[b], 1u)] = i;
}

// The candidate test of two moving bodies: their bounding spheres, grown by both eps,
// overlap.  With skin > 0 the reach is widened by skin (the skin list's build test); with
// skin 0 it is the step's test exactly.  The pair is taken in index order, so the
// rounding of the sums is the same whichever body the search starts from.
__device__ __forceinline__ bool spheres_within(const delta_scene &s, int32_t i0, int32_t j0, double skin) {
  const int32_t n = s.n_bodies;
  const int32_t i = i0 < j0 ? i0 : j0, j = i0 < j0 ? j0 : i0;
  double d2 = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double d = s.pos[(int64_t)k * n + j] - s.pos[(int64_t)k * n + i];
    d2 += d * d;
  }
  double reach = (s.radius[i] + s.radius[j] + s.eps[i] + s.eps[j]) * (1.0 + 1e-9) + 1e-12;
  if (skin > 0.0) reach = (reach + skin) * (1.0 + 1e-9) + 1e-12;
  return d2 <= reach * reach;
}

__device__ __forceinline__ bool spheres_touch(const delta_scene &s, int32_t i, int32_t j) {
  return spheres_within(s, i, j, 0.0);
}

// The candidate test of obstacle L (box lo[3], hi[3]) and moving body j: the body's centre
// within its radius and both eps of the box; skin as in spheres_within.
__device__ __forceinline__ bool obstacle_within(const delta_scene &s, const double *box, int32_t L, int32_t j,
                                                double skin) {
  double d2 = 0.0;
  for (int k = 0; k < 3; ++k) {
    const double c = s.pos[(int64_t)k * s.n_bodies + j];
    const double lo = box[k], hi = box[3 + k];
    const double d = c < lo ? lo - c : (c > hi ? c - hi : 0.0);
    d2 += d * d;
  }
  double reach = (s.radius[j] + s.eps[j] + s.eps[L]) * (1.0 + 1e-9) + 1e-12;
  if (skin > 0.0) reach = (reach + skin) * (1.0 + 1e-9) + 1e-12;
  return d2 <= reach * reach;
}

// pair key (min << sh | max), sh the bits of a body index, so pairs sort in 2*sh bits
__device__ __forceinline__ void push_pair(int32_t a, int32_t b, int sh, uint64_t *out, unsigned long long *count,
                                          int64_t cap) {
  const unsigned long long pos = atomicAdd(count, 1ull);
  if ((int64_t)pos < cap) out[pos] = ((uint64_t)(uint32_t)(a < b ? a : b) << sh) | (uint32_t)(a < b ? b : a);
}

// Each unordered pair is searched from one side only: body i looks at its own cell (for
// bodies j > i) and at the 13 neighbour cells whose offset (dx, dy, dz) is positive in
// lexicographic order (for any body j); a pair in two different cells is met from the body
// whose neighbour offset is positive, exactly once.  Five threads per body, one per cell
// column: (1, -1), (1, 0), (1, 1) and (0, 1) take dz = -1, 0, 1; (0, 0) takes dz = 0 (j > i)
// and 1.  In a cell's bucket a body counts only when its cell key is the cell's; the 27
// neighbour cells have distinct keys and every body one key.  (Cells 2^kCellBits apart
// share keys; their bodies become extra candidates that the sphere test rejects.)  The
// pairs pushed, as (min, max) keys, are those of a search of all 27 cells for j > i.
constexpr int kGridColumns = 5;

__global__ void k_grid_pairs(delta_scene s, Grid g, HashGrid hg, int sh, uint64_t *out, unsigned long long *count,
                             int64_t cap, double skin) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= kGridColumns * (int64_t)s.n_bodies) return;
  const int32_t i = (int32_t)(t / kGridColumns), col = (int32_t)(t % kGridColumns);
  if (s.obstacle[i]) return;
  // the body's cell from the key the count pass stored (coordinates modulo 2^kCellBits,
  // which is all cell_key keeps), instead of three FP64 divisions per thread
  const uint64_t own = hg.cell[i];
  const int64_t c[3] = {(int64_t)((own >> (2 * kCellBits)) & kCellMask), (int64_t)((own >> kCellBits) & kCellMask),
                        (int64_t)(own & kCellMask)};
  const int dx = col < 3 ? 1 : 0, dy = col < 3 ? col - 1 : (col == 3 ? 1 : 0);
  const int dz0 = col == 4 ? 0 : -1;
  const int64_t cx = c[0] + dx, cy = c[1] + dy;
  for (int dz = dz0; dz <= 1; ++dz) {
    const bool same = col == 4 && dz == 0;  // the body's own cell: only j > i
    const uint64_t key = cell_key(cx, cy, c[2] + dz);
    const uint32_t b = cell_bucket(key, hg.nb);
    for (uint32_t q = hg.start[b]; q < hg.start[b + 1]; ++q) {
      const int32_t j = hg.bodies[q];
      if ((same ? j > i : j != i) && hg.cell[j] == key && spheres_within(s, i, j, skin))
        push_pair(i, j, sh, out, count, cap);
    }
  }
}

// obstacle L (box lo/hi) against every moving body j
__global__ void k_obstacle_pairs(delta_scene s, const int32_t *obst, const double *box, int32_t n_obst, int sh,
                                 uint64_t *out, unsigned long long *count, int64_t cap, double skin) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)n_obst * s.n_bodies) return;
  const int32_t o = (int32_t)(t / s.n_bodies), j = (int32_t)(t % s.n_bodies);
  const int32_t L = obst[o];
  if (s.obstacle[j]) return;
  if (obstacle_within(s, box + 6 * o, L, j, skin)) push_pair(L, j, sh, out, count, cap);
}

// The fixed-capacity pair list of at most kBlockSortCap entries, sorted and unpacked by
// one CTA (cub's block radix sort over the 2 sh key bits: 32-bit keys up to 2^16 bodies,
// 64-bit keys above) instead of a device-wide radix sort (a histogram and one launch per
// digit) and an unpacking kernel: one graph node instead of six.  The result, the
// overflow flag and the pair total are k_unpack_pairs's.
constexpr int kBlockSortThreads = 512, kBlockSortItems = 16;
constexpr int64_t kBlockSortCap = (int64_t)kBlockSortThreads * kBlockSortItems;

template <class K, int ITEMS>
using PairBlockSort = cub::BlockRadixSort<K, kBlockSortThreads, ITEMS, cub::NullType, 5>;

// Shared memory of the block sort of up to MAXI keys per thread (the largest variant's).
template <class K, int MAXI>
constexpr size_t block_sort_smem() {
  return sizeof(typename PairBlockSort<K, MAXI>::TempStorage) > sizeof(typename PairBlockSort<K, 2>::TempStorage)
             ? sizeof(typename PairBlockSort<K, MAXI>::TempStorage)
             : sizeof(typename PairBlockSort<K, 2>::TempStorage);
}

// Sorts keys[0 .. m) (m <= 512 * ITEMS) and unpacks them to a, b; entries [m, cap) are
// empty (-1, -1), as the padding keys of a sort over the whole capacity would leave them.
// With kout, the sorted keys go to kout instead ([m, cap) the empty key ~0).
template <class K, int ITEMS>
__device__ __forceinline__ void sort_unpack_items(unsigned char *smem, const uint64_t *__restrict__ keys, int64_t m,
                                                  int64_t cap, int sh, int32_t *__restrict__ a,
                                                  int32_t *__restrict__ b, uint64_t *__restrict__ kout) {
  auto &tmp = *reinterpret_cast<typename PairBlockSort<K, ITEMS>::TempStorage *>(smem);
  const int t = threadIdx.x;
  K k[ITEMS];
#pragma unroll
  for (int j = 0; j < ITEMS; ++j) {
    const int64_t i = (int64_t)t * ITEMS + j;
    // a valid key has a < b < 2^sh, so its 2 sh bits are never all set: the padding
    // key ~0 sorts last
    k[j] = i < m ? (K)keys[i] : ~(K)0;
  }
  PairBlockSort<K, ITEMS>(tmp).Sort(k, 0, 2 * sh);
  if (kout) {
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      const int64_t i = (int64_t)t * ITEMS + j;
      if (i < m) kout[i] = (uint64_t)k[j];
    }
    for (int64_t i = m + t; i < cap; i += kBlockSortThreads) kout[i] = ~0ull;
    return;
  }
  const K low = ((K)1 << sh) - (K)1;
#pragma unroll
  for (int j = 0; j < ITEMS; ++j) {
    const int64_t i = (int64_t)t * ITEMS + j;
    if (i < m) {
      a[i] = (int32_t)(k[j] >> sh);
      b[i] = (int32_t)(k[j] & low);
    }
  }
  for (int64_t i = m + t; i < cap; i += kBlockSortThreads) a[i] = b[i] = -1;
}

// The pair list's block sort, sized at run time to the step's pair count (the smallest
// of 2, 4, 8, 16 keys per thread that holds it, at most MAXI): a sort sized to the
// capacity pays for every padded key (8,192 keys for the hopper's 2,860 pairs).
template <class K, int MAXI>
__global__ void __launch_bounds__(kBlockSortThreads) k_sort_unpack_pairs_block(
    const uint64_t *__restrict__ keys, int64_t cap, int sh, int32_t *__restrict__ a, int32_t *__restrict__ b,
    const unsigned long long *count, int *ovf, int64_t *total, uint64_t *__restrict__ kout) {
  extern __shared__ __align__(16) unsigned char smem[];
  const unsigned long long c = *count;
  if (threadIdx.x == 0) {
    if (c > (unsigned long long)cap) atomicCAS(ovf, 0, 1);
    if (total) *total += (int64_t)(c < (unsigned long long)cap ? c : (unsigned long long)cap);
  }
  const int64_t m = c < (unsigned long long)cap ? (int64_t)c : cap;
  constexpr int T = kBlockSortThreads;
  if (m <= 2 * T) sort_unpack_items<K, 2>(smem, keys, m, cap, sh, a, b, kout);
  else if (m <= 4 * T) sort_unpack_items<K, (MAXI < 4 ? MAXI : 4)>(smem, keys, m, cap, sh, a, b, kout);
  else if (m <= 8 * T) sort_unpack_items<K, (MAXI < 8 ? MAXI : 8)>(smem, keys, m, cap, sh, a, b, kout);
  else sort_unpack_items<K, MAXI>(smem, keys, m, cap, sh, a, b, kout);
}

template <class K, int MAXI>
static cudaError_t block_sort_attr() {
  return cudaFuncSetAttribute(k_sort_unpack_pairs_block<K, MAXI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)block_sort_smem<K, MAXI>());
}

// Raises the dynamic shared memory limit of the block sorts that need more than the
// default 48 KB (called before a capture, outside it).
static cudaError_t block_sort_prepare() {
  cudaError_t e;
  if ((e = block_sort_attr<uint32_t, 16>()) != cudaSuccess) return e;
  if ((e = block_sort_attr<uint64_t, 8>()) != cudaSuccess) return e;
  return block_sort_attr<uint64_t, 16>();
}

template <class K>
static void launch_block_sort(cudaStream_t st, const uint64_t *pk, int64_t cap, int sh, int32_t *pa, int32_t *pb,
                              const unsigned long long *count, int *ovf, int64_t *total, uint64_t *kout = nullptr) {
  constexpr int64_t T = kBlockSortThreads;
  if (cap <= 2 * T)
    k_sort_unpack_pairs_block<K, 2><<<1, T, block_sort_smem<K, 2>(), st>>>(pk, cap, sh, pa, pb, count, ovf, total,
                                                                          kout);
  else if (cap <= 4 * T)
    k_sort_unpack_pairs_block<K, 4><<<1, T, block_sort_smem<K, 4>(), st>>>(pk, cap, sh, pa, pb, count, ovf, total,
                                                                          kout);
  else if (cap <= 8 * T)
    k_sort_unpack_pairs_block<K, 8><<<1, T, block_sort_smem<K, 8>(), st>>>(pk, cap, sh, pa, pb, count, ovf, total,
                                                                          kout);
  else
    k_sort_unpack_pairs_block<K, 16><<<1, T, block_sort_smem<K, 16>(), st>>>(pk, cap, sh, pa, pb, count, ovf, total,
                                                                            kout);
}

// pair keys back to (a, b); the empty key ~0 gives (-1, -1).  With `count` (fixed
// capacity n), thread 0 also flags an overflow of the n entries and adds the step's
// candidate body pairs to *total.
__global__ void k_unpack_pairs(const uint64_t *k, int64_t n, int sh, int32_t *a, int32_t *b,
                               const unsigned long long *count, int *ovf, int64_t *total) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (count && t == 0) {
    const unsigned long long c = *count;
    if (c > (unsigned long long)n) atomicCAS(ovf, 0, 1);
    if (total) *total += (int64_t)(c < (unsigned long long)n ? c : (unsigned long long)n);
  }
  if (t >= n) return;
  const uint64_t v = k[t];
  const bool empty = v == ~0ull;
  a[t] = empty ? -1 : (int32_t)(v >> sh);
  b[t] = empty ? -1 : (int32_t)(v & ((1ull << sh) - 1));
}

// ---- the reference's per-call forces and dynamics, batched --------------------------
// getContactsForces (forces.cpp:291-396) for group g: the contacts [off[g], off[g+1]) of
// body A against body B, added in list order onto force[g], torque[g] (3 planes of n).
struct GroupKin {
  const double *pos_a, *ang_a, *lin_a, *mass_a, *pos_b, *ang_b, *lin_b, *mass_b;
};
__global__ void k_contact_forces_groups(int64_t n, const int64_t *off, ContactView cv, GroupKin g,
                                        delta_step_params p, double *force, double *torque) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  BodyKin A, B;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    A.pos[d] = X(g.pos_a[d * n + i]);
    A.ang[d] = X(g.ang_a[d * n + i]);
    A.lin[d] = X(g.lin_a[d * n + i]);
    B.pos[d] = X(g.pos_b[d * n + i]);
    B.ang[d] = X(g.ang_b[d * n + i]);
    B.lin[d] = X(g.lin_b[d * n + i]);
  }
  A.mass = X(g.mass_a[i]);
  B.mass = X(g.mass_b[i]);
  X F[3], T[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    F[d] = X(force[d * n + i]);
    T[d] = X(torque[d * n + i]);
  }
  const int64_t c0 = max((int64_t)0, off[i]), c1 = min(cv.cap, off[i + 1]);
  for (int64_t c = c0; c < c1; ++c) {
    X Fc[3], Tc[3];
    contact_terms(cv, c, A, B, false, p, Fc, Tc);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      F[d] += Fc[d];
      T[d] += Tc[d];
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    force[d * n + i] = F[d].v;
    torque[d * n + i] = T[d].v;
  }
}

// updateAngular (dynamics.cpp:140-213) of every body of s with its torque (3 planes).
__global__ void k_update_angular_only(delta_scene s, const double *torque, double step) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n_bodies) return;
  const BodyRef b{s.n_bodies, i};
  X tq[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) tq[k] = X(torque[b.at(k)]);
  update_angular(s, b, tq, X(step));
}

// updateRotationMatrix (dynamics.cpp:104-138) of every body of s.
__global__ void k_update_rotation_only(delta_scene s, double step) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n_bodies) return;
  update_rotation(s, BodyRef{s.n_bodies, i}, X(step));
}

// updateVertices (dynamics.cpp:215-242) of vertex v, owned by body[v] of n bodies.
__global__ void k_update_vertices_only(int64_t nv, const int32_t *body, int32_t n, double *x, double *y, double *z,
                                       const double *rx, const double *ry, const double *rz, const double *rot,
                                       const double *pos, const double *ref_pos) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  const int32_t i = body ? body[v] : 0;
  if (i < 0 || i >= n) return;
  xf64 R[9], P[3], RP[3];
#pragma unroll
  for (int k = 0; k < 9; ++k) R[k] = xf64(rot[(int64_t)k * n + i]);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    P[k] = xf64(pos[(int64_t)k * n + i]);
    RP[k] = xf64(ref_pos[(int64_t)k * n + i]);
  }
  double out[3];
  posed_point(R, P, RP, rx[v], ry[v], rz[v], out);
  x[v] = out[0];
  y[v] = out[1];
  z[v] = out[2];
}

__global__ void k_iota32(int32_t *v, int32_t n) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = i;
}

inline unsigned blocks_for(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t > 0 ? (n + t - 1) / t : 1); }

}  // namespace

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------

// Buffers owned by a force evaluation (context scratch slots 7..9).
delta_status forces_run(delta_ctx *ctx, const delta_scene &s, const delta_contacts &c, int64_t n_contacts,
                        const delta_step_params &p, double *force, double *torque, uint8_t *has) {
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  delta_status ds;
  const int32_t n = s.n_bodies;
  if (n_contacts == 0) {
    if ((e = cudaMemsetAsync(force, 0, sizeof(double) * 3 * n, st)) != cudaSuccess ||
        (e = cudaMemsetAsync(torque, 0, sizeof(double) * 3 * n, st)) != cudaSuccess ||
        (e = cudaMemsetAsync(has, 0, (size_t)n, st)) != cudaSuccess)
      return cuda_error(e, "forces memset");
    return DELTA_OK;
  }
  ContactView cv{c.x, c.normal, c.depth, c.master, c.slave, c.friction, c.capacity};
  // scratch: segment count, segment starts (nc), entry keys and sorted keys, entry
  // indices and sorted indices (2 nc each: two entries per segment), entries (2 nc x 6
  // doubles), head flags (nc bytes); the size is the sum of the same terms
  const size_t nc = (size_t)n_contacts;
  const size_t off_seg = 64, off_key = off_seg + 8 * nc, off_skey = off_key + 16 * nc, off_idx = off_skey + 16 * nc,
               off_sidx = off_idx + 16 * nc, off_entry = off_sidx + 16 * nc, off_head = off_entry + 96 * nc,
               bytes = off_head + nc;
  void *buf = nullptr;
  if ((ds = ctx_scratch(ctx, 7, bytes, &buf)) != DELTA_OK) return ds;
  char *b = (char *)buf;
  int64_t *n_seg = (int64_t *)b;
  int64_t *seg_start = (int64_t *)(b + off_seg);
  uint64_t *key = (uint64_t *)(b + off_key);
  uint64_t *skey = (uint64_t *)(b + off_skey);
  int64_t *idx = (int64_t *)(b + off_idx);
  int64_t *sidx = (int64_t *)(b + off_sidx);
  double *entry = (double *)(b + off_entry);
  uint8_t *head = (uint8_t *)(b + off_head);
  k_segment_heads<<<blocks_for(n_contacts), 256, 0, st>>>(cv, n_contacts, head);
  ctx->launches += 1;
  // segment starts: indices where head == 1
  size_t tb = 0;
  cub::CountingInputIterator<int64_t> it(0);
  cub::DeviceSelect::Flagged(nullptr, tb, it, head, seg_start, n_seg, n_contacts, st);
  void *temp = nullptr;
  if ((ds = ctx_scratch(ctx, 8, tb, &temp)) != DELTA_OK) return ds;
  if ((e = cub::DeviceSelect::Flagged(temp, tb, it, head, seg_start, n_seg, n_contacts, st)) != cudaSuccess)
    return cuda_error(e, "segment select");
  ctx->launches += 1;
  // entries for all potential segments (n_contacts bounds the count; unused keys sort last)
  if ((e = cudaMemsetAsync(key, 0xff, sizeof(uint64_t) * 2 * nc, st)) != cudaSuccess) return cuda_error(e, "memset");
  const int sh = bits_for(n);
  k_pair_forces_heads<false><<<blocks_for(n_contacts, kHeadThreads), kHeadThreads, 0, st>>>(
      s, cv, nullptr, n_contacts, seg_start, n_seg, p, sh, key, idx, entry, nullptr);
  ctx->launches += 1;
  tb = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, key, skey, idx, sidx, (int64_t)(2 * nc), 0, 2 * sh, st);
  if ((ds = ctx_scratch(ctx, 8, tb, &temp)) != DELTA_OK) return ds;
  if ((e = cub::DeviceRadixSort::SortPairs(temp, tb, key, skey, idx, sidx, (int64_t)(2 * nc), 0, 2 * sh, st)) !=
      cudaSuccess)
    return cuda_error(e, "entry sort");
  ctx->launches += 1;
  if ((e = zero_body_sums(st, n, force, torque, has)) != cudaSuccess) return cuda_error(e, "forces memset");
  k_body_forces<<<blocks_for((int64_t)(2 * nc)), 256, 0, st>>>(n, sh, skey, sidx, entry, (int64_t)(2 * nc), force,
                                                               torque, has);
  ctx->launches += 1;
  return DELTA_OK;
}

delta_status integrate_run(delta_ctx *ctx, const delta_scene &s, const delta_step_params &p, const double *force,
                           const double *torque, const uint8_t *has, int64_t n_vertices) {
  cudaStream_t st = ctx->stream;
  k_bodies<<<blocks_for(s.n_bodies, 128), 128, 0, st>>>(s, p, force, torque, has, nullptr, nullptr, nullptr);
  (void)n_vertices;
  k_vertices<<<vertex_blocks(s.n_bodies), 256, 0, st>>>(s, nullptr, nullptr, nullptr, nullptr);
  ctx->launches += 2;
  return cuda_error(cudaGetLastError(), "integrate launch");
}

// Grid and obstacle boxes of a scene.  Obstacles are static: their boxes are computed
// once from their current vertices.
struct BroadphasePlan {
  Grid g{};
  // the graph step's skin list: pairs within reach + skin, searched on the grid gs whose
  // cells hold that reach (0: no skin list)
  double skin = 0.0;
  Grid gs{};
  int32_t n_obst = 0, n_moving = 0;
  int32_t *d_obst = nullptr;  // obstacle body indices
  double *d_box = nullptr;    // [6*n_obst] lo(3) hi(3)
  int32_t *d_slot = nullptr;  // [n] each body's obstacle index o (its box at d_box + 6 o), -1 if moving
  void release() {
    if (d_obst) cudaFree(d_obst);
    if (d_box) cudaFree(d_box);
    if (d_slot) cudaFree(d_slot);
    d_obst = nullptr;
    d_box = nullptr;
    d_slot = nullptr;
  }
};

delta_status broadphase_plan(delta_ctx *ctx, const delta_scene &s, BroadphasePlan &plan) {
  const int32_t n = s.n_bodies;
  cudaError_t e;
  std::vector<double> pos(3 * (size_t)n), rad(n), eps(n);
  std::vector<uint8_t> obst(n);
  std::vector<int64_t> off(n + 1);
  if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess ||
      (e = cudaMemcpy(pos.data(), s.pos, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost)) != cudaSuccess ||
      (e = cudaMemcpy(rad.data(), s.radius, sizeof(double) * n, cudaMemcpyDeviceToHost)) != cudaSuccess ||
      (e = cudaMemcpy(eps.data(), s.eps, sizeof(double) * n, cudaMemcpyDeviceToHost)) != cudaSuccess ||
      (e = cudaMemcpy(obst.data(), s.obstacle, n, cudaMemcpyDeviceToHost)) != cudaSuccess ||
      (e = cudaMemcpy(off.data(), s.tri_offset, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost)) != cudaSuccess)
    return cuda_error(e, "broadphase plan copy");
  double reach = 0.0, lo[3] = {1e300, 1e300, 1e300};
  std::vector<int32_t> ob;
  for (int32_t i = 0; i < n; ++i) {
    if (obst[i]) {
      ob.push_back(i);
      continue;
    }
    reach = std::fmax(reach, rad[i] + eps[i]);
    for (int k = 0; k < 3; ++k) lo[k] = std::fmin(lo[k], pos[(size_t)k * n + i]);
  }
  plan.release();
  plan.g.h = reach > 0 ? 2.0 * reach * (1.0 + 1e-6) : 1.0;
  // cell keys wrap (cell_key), so any origin works; the lowest moving centre is used
  for (int k = 0; k < 3; ++k) plan.g.origin[k] = lo[k] < 1e299 ? lo[k] : 0.0;
  // skin: 1/32 of a cell (a body moves it in far more steps than a call takes in these
  // scenes); its grid's cells hold the widened reach
  plan.skin = reach > 0 ? plan.g.h / kSkinPerCell : 0.0;
  plan.gs = plan.g;
  plan.gs.h = reach > 0 ? (2.0 * reach + plan.skin) * (1.0 + 1e-6) + 1e-9 : 1.0;
  plan.n_obst = (int32_t)ob.size();
  plan.n_moving = n - plan.n_obst;
  if (plan.n_obst > 0) {
    // obstacle boxes from their vertices
    std::vector<double> box(6 * ob.size());
    for (size_t o = 0; o < ob.size(); ++o) {
      const int32_t L = ob[o];
      const int64_t v0 = 3 * off[L], v1 = 3 * off[L + 1];
      std::vector<double> xs(v1 - v0), ys(v1 - v0), zs(v1 - v0);
      if ((e = cudaMemcpy(xs.data(), s.x + v0, sizeof(double) * (v1 - v0), cudaMemcpyDeviceToHost)) != cudaSuccess ||
          (e = cudaMemcpy(ys.data(), s.y + v0, sizeof(double) * (v1 - v0), cudaMemcpyDeviceToHost)) != cudaSuccess ||
          (e = cudaMemcpy(zs.data(), s.z + v0, sizeof(double) * (v1 - v0), cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_error(e, "obstacle vertices");
      double bl[3] = {1e300, 1e300, 1e300}, bh[3] = {-1e300, -1e300, -1e300};
      for (size_t q = 0; q < xs.size(); ++q) {
        const double c[3] = {xs[q], ys[q], zs[q]};
        for (int k = 0; k < 3; ++k) {
          bl[k] = std::fmin(bl[k], c[k]);
          bh[k] = std::fmax(bh[k], c[k]);
        }
      }
      for (int k = 0; k < 3; ++k) {
        box[6 * o + k] = bl[k];
        box[6 * o + 3 + k] = bh[k];
      }
    }
    std::vector<int32_t> slot(n, -1);
    for (size_t o = 0; o < ob.size(); ++o) slot[ob[o]] = (int32_t)o;
    if ((e = cudaMalloc(&plan.d_obst, sizeof(int32_t) * ob.size())) != cudaSuccess ||
        (e = cudaMalloc(&plan.d_box, sizeof(double) * box.size())) != cudaSuccess ||
        (e = cudaMalloc(&plan.d_slot, sizeof(int32_t) * (size_t)n)) != cudaSuccess ||
        (e = cudaMemcpy(plan.d_obst, ob.data(), sizeof(int32_t) * ob.size(), cudaMemcpyHostToDevice)) !=
            cudaSuccess ||
        (e = cudaMemcpy(plan.d_box, box.data(), sizeof(double) * box.size(), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(plan.d_slot, slot.data(), sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice)) != cudaSuccess)
      return cuda_error(e, "obstacle upload");
  }
  return DELTA_OK;
}

// Scratch slots 10 (cell keys), 11 (pair keys), 12 (sort temp).
// Hash grid arrays carved from `base` (256-byte aligned pieces); returns the end.
static char *carve_grid(char *base, int32_t n, HashGrid &hg) {
  auto align = [](char *q) { return (char *)(((uintptr_t)q + 255) & ~(uintptr_t)255); };
  char *b = align(base);
  hg.nb = grid_buckets(n);
  hg.count = (uint32_t *)b;
  hg.fill = hg.count + hg.nb + 1;  // zeroed together with count
  b = align(b + 4 * (2 * (size_t)hg.nb + 1));
  hg.start = (uint32_t *)b;
  b = align(b + 4 * ((size_t)hg.nb + 1));
  hg.bodies = (int32_t *)b;
  b = align(b + 4 * (size_t)n);
  hg.cell = (uint64_t *)b;
  return align(b + 8 * (size_t)n);
}

static size_t grid_bytes(int32_t n) {
  const size_t nb = (size_t)grid_buckets(n);
  return 5 * 256 + 4 * (2 * nb + 1) + 4 * (nb + 1) + 12 * (size_t)n;
}

// count, scan, fill: the hash grid of the moving bodies (count and fill zeroed first)
static cudaError_t build_grid(cudaStream_t st, const delta_scene &s, const Grid &grid, const HashGrid &hg,
                              void *temp, size_t temp_bytes, uint64_t *pk, int64_t pk_cap, unsigned long long *pcount) {
  const int32_t n = s.n_bodies;
  cudaError_t e = cudaMemsetAsync(hg.count, 0, 4 * (2 * (size_t)hg.nb + 1), st);
  if (e != cudaSuccess) return e;
  k_grid_count<<<blocks_for(n), 256, 0, st>>>(s, grid, hg, pk, pk_cap, pcount);
  size_t tb = temp_bytes;
  if ((e = exclusive_sum(temp, tb, hg.count, hg.start, hg.nb + 1, st)) != cudaSuccess) return e;
  k_grid_fill<<<blocks_for(n), 256, 0, st>>>(s, hg);
  return cudaGetLastError();
}

static size_t grid_temp_bytes(int32_t n) {
  size_t tb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb, (uint32_t *)nullptr, (uint32_t *)nullptr, grid_buckets(n) + 1);
  return tb;
}

delta_status broadphase_run(delta_ctx *ctx, const delta_scene &s, const BroadphasePlan &plan, int32_t *pair_a,
                            int32_t *pair_b, int64_t capacity, int64_t *n_out) {
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  delta_status ds;
  const int32_t n = s.n_bodies;
  const int sh = bits_for(n);
  void *kb = nullptr;
  if ((ds = ctx_scratch(ctx, 10, grid_bytes(n), &kb)) != DELTA_OK) return ds;
  HashGrid hg{};
  carve_grid((char *)kb, n, hg);
  size_t tb = grid_temp_bytes(n);
  void *temp = nullptr;
  if ((ds = ctx_scratch(ctx, 12, tb, &temp)) != DELTA_OK) return ds;
  if ((e = build_grid(st, s, plan.g, hg, temp, tb, nullptr, 0, nullptr)) != cudaSuccess) return cuda_error(e, "grid");
  ctx->launches += 3;
  int64_t cap = capacity > 4096 ? capacity : 4096;
  unsigned long long hcount = 0;
  uint64_t *pk = nullptr;
  for (int attempt = 0; attempt < 2; ++attempt) {
    void *pb = nullptr;
    if ((ds = ctx_scratch(ctx, 11, sizeof(uint64_t) * 2 * (size_t)cap + 64, &pb)) != DELTA_OK) return ds;
    unsigned long long *count = (unsigned long long *)pb;
    pk = (uint64_t *)pb + 8;
    if ((e = cudaMemsetAsync(count, 0, sizeof(unsigned long long), st)) != cudaSuccess) return cuda_error(e, "memset");
    if (plan.n_moving > 0) {
      k_grid_pairs<<<blocks_for(kGridColumns * (int64_t)n, 128), 128, 0, st>>>(s, plan.g, hg, sh, pk, count, cap,
                                                                                0.0);
      ctx->launches += 1;
    }
    if (plan.n_obst > 0) {
      k_obstacle_pairs<<<blocks_for((int64_t)plan.n_obst * n), 256, 0, st>>>(s, plan.d_obst, plan.d_box, plan.n_obst,
                                                                            sh, pk, count, cap, 0.0);
      ctx->launches += 1;
    }
    if ((e = cudaMemcpyAsync(&hcount, count, sizeof(hcount), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
      return cuda_error(e, "broadphase count");
    if ((int64_t)hcount <= cap) break;
    cap = (int64_t)hcount + hcount / 2;
  }
  const int64_t np = (int64_t)hcount;
  *n_out = np;
  if (np == 0) return DELTA_OK;
  uint64_t *spk = pk + cap;
  tb = 0;
  cub::DeviceRadixSort::SortKeys(nullptr, tb, pk, spk, np, 0, 2 * sh, st);
  if ((ds = ctx_scratch(ctx, 12, tb, &temp)) != DELTA_OK) return ds;
  if ((e = cub::DeviceRadixSort::SortKeys(temp, tb, pk, spk, np, 0, 2 * sh, st)) != cudaSuccess)
    return cuda_error(e, "pair sort");
  ctx->launches += 1;
  const int64_t wn = np < capacity ? np : capacity;
  if (wn > 0) {
    k_unpack_pairs<<<blocks_for(wn), 256, 0, st>>>(spk, wn, sh, pair_a, pair_b, nullptr, nullptr, nullptr);
    ctx->launches += 1;
  }
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_error(e, "broadphase");
  if (np > capacity) return set_error(DELTA_ERR_CAPACITY, "delta_broadphase: pair capacity exceeded");
  return DELTA_OK;
}


// Forces from a fixed-capacity contact buffer with its count on the device.
size_t forces_fixed_state_bytes(int64_t cap, int32_t n_bodies) {
  return 4 * 256 + 96 * (size_t)cap + 4 * (size_t)cap + 4 * (2 * (size_t)n_bodies + 1) + 4 * ((size_t)n_bodies + 1);
}

size_t forces_fixed_temp_bytes(int64_t cap, int32_t n_bodies) {
  (void)cap;
  size_t b = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, b, (uint32_t *)nullptr, (uint32_t *)nullptr, (int64_t)n_bodies + 1);
  return b;
}

// The fixed-capacity force state: entries (2 per segment, 6 doubles), slave lists, slave
// counts [n + 1] and fill positions [n] (adjacent), list starts [n + 1].
static void forces_fixed_layout(void *state, int64_t cap, int32_t n, double *&entry, int32_t *&list, uint32_t *&cnt,
                                uint32_t *&fill, uint32_t *&start) {
  auto align = [](char *q) { return (char *)(((uintptr_t)q + 255) & ~(uintptr_t)255); };
  char *b = align((char *)state);
  entry = (double *)b;
  b = align(b + 96 * (size_t)cap);
  list = (int32_t *)b;
  b = align(b + 4 * (size_t)cap);
  cnt = (uint32_t *)b;
  fill = cnt + n + 1;
  b = align(b + 4 * (2 * (size_t)n + 1));
  start = (uint32_t *)b;
}

// Once per allocation of the force state: slave counts and fill positions at zero.
static cudaError_t forces_fixed_init(cudaStream_t st, void *state, int64_t cap, int32_t n) {
  double *entry;
  int32_t *list;
  uint32_t *cnt, *fill, *start;
  forces_fixed_layout(state, cap, n, entry, list, cnt, fill, start);
  return cudaMemsetAsync(cnt, 0, 4 * (2 * (size_t)n + 1), st);
}

delta_status forces_run_fixed(cudaStream_t st, const delta_scene &s, const delta_contacts &c, const int64_t *d_nc,
                              const delta_step_params &p, double *force, double *torque, uint8_t *has, void *state,
                              void *temp, size_t temp_bytes, int &kernels) {
  cudaError_t e;
  const int64_t cap = c.capacity;
  const int32_t n = s.n_bodies;
  ContactView cv{c.x, c.normal, c.depth, c.master, c.slave, c.friction, cap};
  double *entry;
  int32_t *list;
  uint32_t *cnt, *fill, *start;
  forces_fixed_layout(state, cap, n, entry, list, cnt, fill, start);
  // cnt and fill are zero: cleared at allocation (forces_fixed_init) and by the per-body
  // sums of the step before
  k_pair_forces_heads<true><<<blocks_for(cap, kHeadThreads), kHeadThreads, 0, st>>>(
      s, cv, d_nc, 0, nullptr, nullptr, p, 0, nullptr, nullptr, entry, cnt);
  size_t tb = temp_bytes;
  // the kernels after the first start as programmatic dependent launches (pdl.cuh)
  if ((e = exclusive_sum(temp, tb, cnt, start, (int64_t)n + 1, st, true)) != cudaSuccess)
    return cuda_error(e, "slave list scan");
  if ((e = launch_dep(true, k_fill_slave_lists, blocks_for(cap), 256, 0, st, s, cv, d_nc, start, fill, list)) !=
          cudaSuccess ||
      (e = launch_dep(true, k_body_forces_lists, blocks_for(n), 256, 0, st, s, cv, d_nc, start, list, entry, force,
                      torque, has, cnt, fill)) != cudaSuccess)
    return cuda_error(e, "forces fixed");
  kernels += 4;
  return cuda_error(cudaGetLastError(), "forces fixed");
}

// Broadphase into a fixed-capacity pair list (padded with -1), overflow flagged on the device.
size_t broadphase_fixed_state_bytes(int32_t n, int64_t pair_cap) {
  return grid_bytes(n) + 512 + (size_t)pair_cap * 16 + 256;
}

size_t broadphase_fixed_temp_bytes(int32_t n, int64_t pair_cap) {
  size_t a = grid_temp_bytes(n), b = 0;
  cub::DeviceRadixSort::SortKeys(nullptr, b, (uint64_t *)nullptr, (uint64_t *)nullptr, pair_cap, 0,
                                 2 * bits_for(n));
  return a > b ? a : b;
}

delta_status broadphase_run_fixed(cudaStream_t st, const delta_scene &s, const BroadphasePlan &plan, int32_t *pair_a,
                                  int32_t *pair_b, int64_t pair_cap, int *ovf, int64_t *pairs_total, void *state,
                                  void *temp, size_t temp_bytes, int &kernels) {
  cudaError_t e;
  const int32_t n = s.n_bodies;
  const int sh = bits_for(n);
  HashGrid hg{};
  char *b = carve_grid((char *)state, n, hg);
  unsigned long long *count = (unsigned long long *)b;
  uint64_t *pk = (uint64_t *)(b + 256), *spk = pk + pair_cap;
  if ((e = build_grid(st, s, plan.g, hg, temp, temp_bytes, pk, pair_cap, count)) != cudaSuccess)
    return cuda_error(e, "grid");
  size_t tb = temp_bytes;
  kernels += 3;
  if (plan.n_moving > 0) {
    k_grid_pairs<<<blocks_for(kGridColumns * (int64_t)n, 128), 128, 0, st>>>(s, plan.g, hg, sh, pk, count, pair_cap,
                                                                                0.0);
    kernels += 1;
  }
  if (plan.n_obst > 0) {
    k_obstacle_pairs<<<blocks_for((int64_t)plan.n_obst * n), 256, 0, st>>>(s, plan.d_obst, plan.d_box, plan.n_obst,
                                                                          sh, pk, count, pair_cap, 0.0);
    kernels += 1;
  }
  if (pair_cap <= kBlockSortCap) {
    if (2 * sh <= 32) launch_block_sort<uint32_t>(st, pk, pair_cap, sh, pair_a, pair_b, count, ovf, pairs_total);
    else launch_block_sort<uint64_t>(st, pk, pair_cap, sh, pair_a, pair_b, count, ovf, pairs_total);
    kernels += 1;
    return cuda_error(cudaGetLastError(), "broadphase fixed");
  }
  tb = temp_bytes;
  if ((e = cub::DeviceRadixSort::SortKeys(temp, tb, pk, spk, pair_cap, 0, 2 * sh, st)) != cudaSuccess)
    return cuda_error(e, "pair sort");
  k_unpack_pairs<<<blocks_for(pair_cap), 256, 0, st>>>(spk, pair_cap, sh, pair_a, pair_b, count, ovf, pairs_total);
  kernels += 2;
  return cuda_error(cudaGetLastError(), "broadphase fixed");
}

// The raw pair count of the last fixed broadphase (for growing the capacity).
static unsigned long long *broadphase_fixed_count(void *state, int32_t n) {
  HashGrid hg{};
  return (unsigned long long *)carve_grid((char *)state, n, hg);
}

// ---- skin list (graph step) ------------------------------------------------------------
// The candidate pairs of a step are those within reach (spheres_touch, obstacle_within).
// The graph step keeps the sorted list of pairs within reach + skin, built at anchor
// positions, and filters it with the exact tests each step, in key order: the same pairs,
// in the same order, as a grid search of that step.  A pair within reach now was within
// reach + skin at the build if neither body has moved more than skin/2 since (triangle
// inequality; the build test's relative and absolute margins cover the rounding), so the
// list is rebuilt, inside the graph through a conditional node, in any step where some
// moving body has moved further.  Obstacles do not move.
struct SkinList {
  int64_t cap = 0;                          // entries of keys, raw, sel
  unsigned long long *raw_count = nullptr;  // pairs found by the last build (may exceed cap)
  int64_t *sel_count = nullptr;             // this step's pairs (multi-CTA filter)
  int *need = nullptr;                      // nonzero: rebuild before this step's filter
  unsigned long long *rebuilds = nullptr;   // builds run inside the graph
  uint64_t *keys = nullptr;                 // [cap] sorted keys of the last build, ~0 after them
  uint64_t *raw = nullptr;                  // [cap] a build's keys as found
  uint64_t *sel = nullptr;                  // [cap] this step's keys (multi-CTA filter)
  double *anchor = nullptr;                 // [3n] positions at the last build
};

static size_t skin_bytes(int32_t n, int64_t cap) { return 256 + 24 * (size_t)cap + 24 * (size_t)n; }

static SkinList carve_skin(void *mem, int32_t n, int64_t cap) {
  SkinList k;
  char *b = (char *)mem;
  k.cap = cap;
  k.raw_count = (unsigned long long *)b;
  k.sel_count = (int64_t *)(b + 8);
  k.rebuilds = (unsigned long long *)(b + 16);
  k.need = (int *)(b + 24);
  k.keys = (uint64_t *)(b + 256);
  k.raw = k.keys + cap;
  k.sel = k.raw + cap;
  k.anchor = (double *)(k.sel + cap);
  (void)n;
  return k;
}

// A pair key of the list (~0: empty) within reach at the current positions.
struct SkinTouch {
  delta_scene s;
  int sh;
  const int32_t *slot;
  const double *box;
  __device__ __forceinline__ bool operator()(uint64_t key) const {
    if (key == ~0ull) return false;
    const int32_t a = (int32_t)(key >> sh), b = (int32_t)(key & ((1ull << sh) - 1ull));
    if (s.obstacle[a]) return obstacle_within(s, box + 6 * slot[a], a, b, 0.0);
    if (s.obstacle[b]) return obstacle_within(s, box + 6 * slot[b], b, a, 0.0);
    return spheres_touch(s, a, b);
  }
};

// Sets *need when a moving body has moved more than `limit` from its anchor (or its
// position is not finite).
__global__ void k_skin_check(delta_scene s, const double *__restrict__ anchor, double limit2, int *need) {
  dep_sync();
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n_bodies || s.obstacle[i]) return;
  const int64_t n = s.n_bodies;
  double d2 = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double d = s.pos[k * n + i] - anchor[k * n + i];
    d2 += d * d;
  }
  if (!(d2 <= limit2)) *need = 1;
}

__global__ void k_skin_cond(cudaGraphConditionalHandle h, const int *need) {
  dep_sync();
  cudaGraphSetConditional(h, *need != 0 ? 1u : 0u);
}

// End of a build: no rebuild pending, one more build counted.
__global__ void k_skin_done(int *need, unsigned long long *rebuilds) {
  *need = 0;
  *rebuilds += 1ull;
}

__global__ void k_skin_overflow(const unsigned long long *raw_count, int64_t cap, int *ovf) {
  if (*raw_count > (unsigned long long)cap) atomicCAS(ovf, 0, 1);
}

// The exact test of every list entry, one thread per entry (the tests' dependent loads
// spread over the GPU): flags[i] = 1 where keys[i] is a pair within reach.
__global__ void k_skin_flags(const uint64_t *__restrict__ keys, int64_t cap, SkinTouch touch,
                             uint8_t *__restrict__ flags) {
  dep_sync();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < cap) flags[i] = touch(keys[i]) ? 1 : 0;
}

// One CTA: the flagged keys of a list of at most 512 * ITEMS entries, in order, into the
// step's pair list (-1 after the pairs); *count_out receives the pairs found, an overflow
// of pair_cap sets *ovf, *total adds the pairs kept.
template <int ITEMS>
__global__ void __launch_bounds__(kBlockSortThreads) k_skin_compact_block(const uint64_t *__restrict__ keys,
                                                                        const uint8_t *__restrict__ flags, int64_t cap,
                                                                        int sh, int32_t *__restrict__ pa,
                                                                        int32_t *__restrict__ pb, int64_t pair_cap,
                                                                        unsigned long long *count_out, int *ovf,
                                                                        int64_t *total) {
  dep_sync();
  using Scan = cub::BlockScan<int, kBlockSortThreads>;
  __shared__ typename Scan::TempStorage tmp;
  const int t = threadIdx.x;
  uint64_t k[ITEMS];
  int f[ITEMS], pos[ITEMS];
#pragma unroll
  for (int j = 0; j < ITEMS; ++j) {
    const int64_t i = (int64_t)t * ITEMS + j;
    f[j] = i < cap ? flags[i] : 0;
    k[j] = f[j] ? keys[i] : 0ull;
  }
  int found = 0;
  Scan(tmp).ExclusiveSum(f, pos, found);
  const uint64_t low = (1ull << sh) - 1ull;
#pragma unroll
  for (int j = 0; j < ITEMS; ++j)
    if (f[j] && pos[j] < pair_cap) {
      pa[pos[j]] = (int32_t)(k[j] >> sh);
      pb[pos[j]] = (int32_t)(k[j] & low);
    }
  for (int64_t i = found + t; i < pair_cap; i += kBlockSortThreads) pa[i] = pb[i] = -1;
  if (t == 0) {
    *count_out = (unsigned long long)found;
    if (found > pair_cap) atomicCAS(ovf, 0, 1);
    if (total) *total += found < pair_cap ? found : pair_cap;
  }
}

// The multi-CTA filter's output (cub's select, in order) into the step's pair list.
__global__ void k_unpack_selected(const uint64_t *__restrict__ sel, const int64_t *sel_count, int64_t pair_cap, int sh,
                                  int32_t *__restrict__ pa, int32_t *__restrict__ pb, unsigned long long *count_out,
                                  int *ovf, int64_t *total) {
  dep_sync();
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t c = *sel_count;
  if (t == 0) {
    *count_out = (unsigned long long)c;
    if (c > pair_cap) atomicCAS(ovf, 0, 1);
    if (total) *total += c < pair_cap ? c : pair_cap;
  }
  if (t >= pair_cap) return;
  if (t < c) {
    const uint64_t k = sel[t];
    pa[t] = (int32_t)(k >> sh);
    pb[t] = (int32_t)(k & ((1ull << sh) - 1ull));
  } else {
    pa[t] = pb[t] = -1;
  }
}

static SkinTouch skin_touch(const delta_scene &s, const BroadphasePlan &plan) {
  return SkinTouch{s, bits_for(s.n_bodies), plan.d_slot, plan.d_box};
}

// cub's temporary storage for a build's sort and a step's selection over cap entries.
static size_t skin_temp_bytes(const delta_scene &s, const BroadphasePlan &plan, int64_t cap) {
  size_t a = grid_temp_bytes(s.n_bodies), b = 0, c = 0;
  cub::DeviceRadixSort::SortKeys(nullptr, b, (uint64_t *)nullptr, (uint64_t *)nullptr, cap, 0,
                                 2 * bits_for(s.n_bodies));
  cub::DeviceSelect::If(nullptr, c, (const uint64_t *)nullptr, (uint64_t *)nullptr, (int64_t *)nullptr, cap,
                        skin_touch(s, plan));
  return std::max(a, std::max(b, c));
}

// The pairs within reach + skin at the current positions, counted (synchronous; the
// grid part of the fixed broadphase state and its temporary storage are used).
static delta_status skin_count(cudaStream_t st, const delta_scene &s, const BroadphasePlan &plan, void *state,
                               void *temp, size_t temp_bytes, int64_t *found) {
  const int32_t n = s.n_bodies;
  const int sh = bits_for(n);
  HashGrid hg{};
  unsigned long long *count = (unsigned long long *)carve_grid((char *)state, n, hg);
  cudaError_t e;
  if ((e = build_grid(st, s, plan.gs, hg, temp, temp_bytes, nullptr, 0, nullptr)) != cudaSuccess ||
      (e = cudaMemsetAsync(count, 0, sizeof(unsigned long long), st)) != cudaSuccess)
    return cuda_error(e, "skin count");
  if (plan.n_moving > 0)
    k_grid_pairs<<<blocks_for(kGridColumns * (int64_t)n, 128), 128, 0, st>>>(s, plan.gs, hg, sh, nullptr, count, 0,
                                                                            plan.skin);
  if (plan.n_obst > 0)
    k_obstacle_pairs<<<blocks_for((int64_t)plan.n_obst * n), 256, 0, st>>>(s, plan.d_obst, plan.d_box, plan.n_obst,
                                                                          sh, nullptr, count, 0, plan.skin);
  unsigned long long h = 0;
  if ((e = cudaGetLastError()) != cudaSuccess ||
      (e = cudaMemcpyAsync(&h, count, sizeof(h), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return cuda_error(e, "skin count");
  *found = (int64_t)h;
  return DELTA_OK;
}

// A build of the list at the current positions (the body of the graph's conditional
// node): grid on gs, search with the widened reach, sort, anchors; an overflow of the
// capacity sets *ovf.
static cudaError_t skin_build(cudaStream_t st, const delta_scene &s, const BroadphasePlan &plan, const SkinList &k,
                              void *state, void *temp, size_t temp_bytes, int *ovf, int &kernels) {
  const int32_t n = s.n_bodies;
  const int sh = bits_for(n);
  HashGrid hg{};
  carve_grid((char *)state, n, hg);
  cudaError_t e;
  if ((e = build_grid(st, s, plan.gs, hg, temp, temp_bytes, k.raw, k.cap, k.raw_count)) != cudaSuccess) return e;
  kernels += 3;
  if (plan.n_moving > 0) {
    k_grid_pairs<<<blocks_for(kGridColumns * (int64_t)n, 128), 128, 0, st>>>(s, plan.gs, hg, sh, k.raw, k.raw_count,
                                                                            k.cap, plan.skin);
    kernels += 1;
  }
  if (plan.n_obst > 0) {
    k_obstacle_pairs<<<blocks_for((int64_t)plan.n_obst * n), 256, 0, st>>>(s, plan.d_obst, plan.d_box, plan.n_obst,
                                                                          sh, k.raw, k.raw_count, k.cap, plan.skin);
    kernels += 1;
  }
  if (k.cap <= kBlockSortCap) {
    if (2 * sh <= 32) launch_block_sort<uint32_t>(st, k.raw, k.cap, sh, nullptr, nullptr, k.raw_count, ovf, nullptr, k.keys);
    else launch_block_sort<uint64_t>(st, k.raw, k.cap, sh, nullptr, nullptr, k.raw_count, ovf, nullptr, k.keys);
    kernels += 1;
  } else {
    size_t tb = temp_bytes;
    if ((e = cub::DeviceRadixSort::SortKeys(temp, tb, k.raw, k.keys, k.cap, 0, 2 * sh, st)) != cudaSuccess) return e;
    k_skin_overflow<<<1, 1, 0, st>>>(k.raw_count, k.cap, ovf);
    kernels += 2;
  }
  if ((e = cudaMemcpyAsync(k.anchor, s.pos, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToDevice, st)) !=
      cudaSuccess)
    return e;
  k_skin_done<<<1, 1, 0, st>>>(k.need, k.rebuilds);
  kernels += 1;
  return cudaGetLastError();
}

// A step's check: sets the rebuild condition of the graph's conditional node.
static cudaError_t skin_check(cudaStream_t st, const delta_scene &s, const BroadphasePlan &plan, const SkinList &k,
                              cudaGraphConditionalHandle h, int &kernels) {
  const double limit = 0.5 * plan.skin * (1.0 - 1e-9);
  cudaError_t e = launch_dep(true, k_skin_check, blocks_for(s.n_bodies, 256), 256, 0, st, s, k.anchor, limit * limit,
                             k.need);
  if (e == cudaSuccess) e = launch_dep(true, k_skin_cond, 1, 1, 0, st, h, k.need);
  kernels += 2;
  return e;
}

// A step's candidate pairs from the list: the tests one thread per entry and an ordered
// compaction in one CTA for lists of at most kBlockSortCap entries, else cub's select and
// an unpacking kernel.
static cudaError_t skin_filter(cudaStream_t st, const delta_scene &s, const BroadphasePlan &plan, const SkinList &k,
                               int32_t *pa, int32_t *pb, int64_t pair_cap, int *ovf, int64_t *pairs_total, void *state,
                               void *temp, size_t temp_bytes, int &kernels) {
  const SkinTouch touch = skin_touch(s, plan);
  unsigned long long *count_out = broadphase_fixed_count(state, s.n_bodies);
  constexpr int64_t T = kBlockSortThreads;
  if (k.cap <= kBlockSortCap) {
    // the tests on the whole GPU, the ordered compaction in one CTA (the flags in sel)
    uint8_t *flags = reinterpret_cast<uint8_t *>(k.sel);
    // (the flags kernel follows the conditional node: a plain launch)
    k_skin_flags<<<blocks_for(k.cap, 128), 128, 0, st>>>(k.keys, k.cap, touch, flags);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    auto compact = k.cap <= 2 * T   ? k_skin_compact_block<2>
                   : k.cap <= 4 * T ? k_skin_compact_block<4>
                   : k.cap <= 8 * T ? k_skin_compact_block<8>
                                    : k_skin_compact_block<16>;
    kernels += 2;
    return launch_dep(true, compact, 1, (unsigned)T, 0, st, k.keys, flags, k.cap, touch.sh, pa, pb, pair_cap, count_out,
                      ovf, pairs_total);
  } else {
    size_t tb = temp_bytes;
    cudaError_t e = cub::DeviceSelect::If(temp, tb, k.keys, k.sel, k.sel_count, k.cap, touch, st);
    if (e != cudaSuccess) return e;
    kernels += 2;
    return launch_dep(true, k_unpack_selected, blocks_for(pair_cap), 256, 0, st, k.sel, k.sel_count, pair_cap, touch.sh,
                      pa, pb, count_out, ovf, pairs_total);
  }
}
}  // namespace delta

// ---------------------------------------------------------------------------------------
// simulation object
// ---------------------------------------------------------------------------------------

struct delta_sim {
  delta_ctx *ctx = nullptr;
  delta_scene scene{};
  int driver = DELTA_DRV_BF;
  delta::BroadphasePlan plan;
  int64_t n_tri = 0;
  int tri_bits = 16;  // bits of a triangle index within a body (the graph's contact sort keys)
  int32_t *ids = nullptr;
  // Vertex stamps: during a call of several steps only the bodies of each step's candidate
  // pairs get their vertices updated (stamp[i] == *epoch); every vertex is brought up to
  // date at the end of the call.  [n] stamps, then the epoch.
  uint32_t *stamp = nullptr, *epoch = nullptr;
  // The certified driver reads no vertex array during a call: it forms the vertices from
  // the bodies' poses (pose.cuh).  reach: per body, the bound on |r - ref_pos|; obox: the
  // boxes of the obstacles (static), by body.
  double *reach = nullptr, *obox = nullptr;
  // contacts of the last detection
  delta_contacts c{};
  void *c_mem = nullptr;
  int64_t n_contacts = 0;
  // pairs and per-body sums
  int32_t *pa = nullptr, *pb = nullptr;
  int64_t pair_cap = 0;
  double *F = nullptr, *T = nullptr;
  uint8_t *has = nullptr;
  // steps, candidate body pairs, triangle pairs of the candidates, triangle pairs solved
  int64_t counters[4] = {0, 0, 0, 0};
  int64_t graph_pair_cap = 0, graph_contact_cap = 0;  // requested by delta_sim_set_graph_capacity
  int64_t last_pairs = 0;                            // candidate body pairs of the last detection
  int64_t skin_rebuilds = 0;                         // skin list builds inside graph replays
  // graph mode: fixed-capacity buffers, device-side counts, the captured step
  struct Graph {
    int64_t pair_cap = 0, contact_cap = 0;
    int32_t *pa = nullptr, *pb = nullptr;
    void *bp = nullptr, *fs = nullptr, *ds = nullptr, *temp = nullptr, *c_mem = nullptr, *dev = nullptr;
    size_t temp_bytes = 0;
    delta_contacts c{};
    int64_t *d_nc = nullptr, *d_step = nullptr, *d_cnt = nullptr, *d_log = nullptr;
    int *d_ovf = nullptr, *d_snap = nullptr;
    int64_t *d_bp = nullptr;  // candidate body pairs summed over the replayed steps
    int64_t *d_pend = nullptr;  // the step in flight's pairs, triangle pairs, solved pairs
    int64_t log_len = 0;
    // the skin list (its buffer sk), its rebuilds' kernels, and the stream its conditional
    // body is captured from
    void *sk = nullptr;
    delta::SkinList skin{};
    int rebuild_kernels = 0;
    unsigned long long rebuilds_seen = 0;
    cudaStream_t stream2 = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    delta_step_params params{};
    int kernels = 0;
    int64_t launch_epoch = 0;  // the context's launch shapes the graph was recorded with
    bool captured = false;
  } g;
};

namespace delta {

static delta_status alloc_contacts(delta_sim *s, int64_t cap) {
  if (s->c_mem) cudaFree(s->c_mem);
  s->c_mem = nullptr;
  const size_t per = 14 * sizeof(double) + 5 * sizeof(int32_t) + 1;
  cudaError_t e = cudaMalloc(&s->c_mem, per * (size_t)cap + 256);
  if (e != cudaSuccess) return cuda_error(e, "contact buffer");
  double *d = (double *)s->c_mem;
  s->c.capacity = cap;
  s->c.x = d;
  s->c.normal = d + 3 * cap;
  s->c.P = d + 6 * cap;
  s->c.Q = d + 9 * cap;
  s->c.depth = d + 12 * cap;
  s->c.eps_total = d + 13 * cap;
  int32_t *ip = (int32_t *)(d + 14 * cap);
  s->c.master = ip;
  s->c.slave = ip + cap;
  s->c.tri_a = ip + 2 * cap;
  s->c.tri_b = ip + 3 * cap;
  s->c.penetration = ip + 4 * cap;
  s->c.friction = (uint8_t *)(ip + 5 * cap);
  return DELTA_OK;
}

static delta_status alloc_pairs(delta_sim *s, int64_t cap) {
  if (s->pa) cudaFree(s->pa);
  s->pa = nullptr;
  cudaError_t e = cudaMalloc(&s->pa, sizeof(int32_t) * 2 * (size_t)cap);
  if (e != cudaSuccess) return cuda_error(e, "pair buffer");
  s->pb = s->pa + cap;
  s->pair_cap = cap;
  return DELTA_OK;
}

// updateVertices for every body: the end of a call of delta_sim_step(_graph), after which
// the vertices in memory describe the state (the steps in between update only the bodies of
// their candidate pairs).
static delta_status sim_all_vertices(delta_sim *s, cudaStream_t st) {
  k_vertices<<<vertex_blocks(s->scene.n_bodies), 256, 0, st>>>(s->scene, nullptr, nullptr, nullptr, nullptr);
  s->ctx->launches += 1;
  return cuda_error(cudaGetLastError(), "vertex update");
}

// The poses of the simulation's bodies, for the certified driver.
static Pose sim_pose(const delta_sim *s) {
  const delta_scene &c = s->scene;
  return Pose{c.rx, c.ry, c.rz, c.rot, c.pos, c.ref_pos, c.obstacle, s->reach, s->obox, c.n_bodies};
}

static delta_status sim_detect(delta_sim *s) {
  delta_status ds;
  int64_t np = 0;
  ds = broadphase_run(s->ctx, s->scene, s->plan, s->pa, s->pb, s->pair_cap, &np);
  if (ds == DELTA_ERR_CAPACITY) {
    if ((ds = alloc_pairs(s, np + np / 2 + 1024)) != DELTA_OK) return ds;
    ds = broadphase_run(s->ctx, s->scene, s->plan, s->pa, s->pb, s->pair_cap, &np);
  }
  if (ds != DELTA_OK) return ds;
  s->counters[1] += np;
  s->last_pairs = np;
  // vertices of the bodies the narrowphase reads: formed from the poses by the certified
  // driver, updated here for the others
  const bool posed = s->driver == DELTA_DRV_BF_CERT || s->driver == DELTA_DRV_BF_CULLED || s->driver == DELTA_DRV_LEARNED;
  const Pose pose = sim_pose(s);
  if (!posed) {
    cudaStream_t st = s->ctx->stream;
    k_next_epoch<<<1, 1, 0, st>>>(s->epoch);
    if (np > 0) k_mark_pair_bodies<<<blocks_for(np), 256, 0, st>>>(s->pa, s->pb, np, s->epoch, s->stamp);
    k_vertices<<<vertex_blocks(s->scene.n_bodies), 256, 0, st>>>(s->scene, nullptr, nullptr, s->stamp, s->epoch);
    s->ctx->launches += np > 0 ? 3 : 2;
  }
  delta_meshes m{s->scene.n_bodies, s->scene.tri_offset, s->scene.x, s->scene.y, s->scene.z,
                 s->scene.eps,      s->scene.friction,   s->ids};
  int64_t nc = 0;
  if (np == 0) {
    s->n_contacts = 0;
    return DELTA_OK;
  }
  int64_t cnt[2] = {0, 0};
  ds = detect_run(s->ctx, s->driver, DELTA_F64, m, s->pa, s->pb, np, &s->c, &nc, nullptr, cnt,
                    posed ? &pose : nullptr);
  if (ds == DELTA_ERR_CAPACITY) {
    if ((ds = alloc_contacts(s, nc + nc / 2 + 1024)) != DELTA_OK) return ds;
    cnt[0] = cnt[1] = 0;
    ds = detect_run(s->ctx, s->driver, DELTA_F64, m, s->pa, s->pb, np, &s->c, &nc, nullptr, cnt,
                    posed ? &pose : nullptr);
  }
  s->counters[2] += cnt[0];
  s->counters[3] += cnt[1];
  if (ds != DELTA_OK) return ds;
  s->n_contacts = nc;
  return DELTA_OK;
}

static void graph_release(delta_sim::Graph &g) {
  if (g.exec) cudaGraphExecDestroy(g.exec);
  if (g.graph) cudaGraphDestroy(g.graph);
  g.exec = nullptr;
  g.graph = nullptr;
  g.captured = false;
  for (void *p : {(void *)g.pa, g.bp, g.fs, g.ds, g.temp, g.c_mem, g.dev, g.sk})
    if (p) cudaFree(p);
  g.pa = g.pb = nullptr;
  g.bp = g.fs = g.ds = g.temp = g.c_mem = g.dev = g.sk = nullptr;
  g.skin = delta::SkinList{};
  g.rebuilds_seen = 0;
}

// (Re)allocates the fixed buffers for the given capacities (no capture in progress).
static delta_status graph_alloc(delta_sim *s, int64_t pair_cap, int64_t contact_cap, int64_t log_len) {
  delta_sim::Graph &g = s->g;
  graph_release(g);
  const int32_t n = s->scene.n_bodies;
  g.pair_cap = pair_cap;
  g.contact_cap = contact_cap;
  g.log_len = log_len;
  cudaError_t e;
  size_t t = detect_fixed_temp_bytes(pair_cap, contact_cap);
  t = std::max(t, forces_fixed_temp_bytes(contact_cap, n));
  t = std::max(t, broadphase_fixed_temp_bytes(n, pair_cap));
  g.temp_bytes = t + 256;
  const size_t cbytes = (14 * sizeof(double) + 5 * sizeof(int32_t) + 1) * (size_t)contact_cap + 256;
  if ((e = cudaMalloc(&g.pa, sizeof(int32_t) * 2 * (size_t)pair_cap)) != cudaSuccess ||
      (e = cudaMalloc(&g.bp, broadphase_fixed_state_bytes(n, pair_cap))) != cudaSuccess ||
      (e = cudaMalloc(&g.fs, forces_fixed_state_bytes(contact_cap, n))) != cudaSuccess ||
      (e = cudaMalloc(&g.ds, detect_fixed_state_bytes(pair_cap, contact_cap))) != cudaSuccess ||
      (e = cudaMalloc(&g.temp, g.temp_bytes)) != cudaSuccess || (e = cudaMalloc(&g.c_mem, cbytes)) != cudaSuccess ||
      (e = cudaMalloc(&g.dev, 256 + sizeof(int64_t) * (size_t)log_len)) != cudaSuccess)
    return cuda_error(e, "graph buffers");
  g.pb = g.pa + pair_cap;
  double *d = (double *)g.c_mem;
  const int64_t cap = contact_cap;
  g.c = delta_contacts{cap, d, d + 3 * cap, d + 6 * cap, d + 9 * cap, d + 12 * cap, d + 13 * cap,
                       (int32_t *)(d + 14 * cap), (int32_t *)(d + 14 * cap) + cap,
                       (int32_t *)(d + 14 * cap) + 2 * cap, (int32_t *)(d + 14 * cap) + 3 * cap,
                       (int32_t *)(d + 14 * cap) + 4 * cap, (uint8_t *)((int32_t *)(d + 14 * cap) + 5 * cap)};
  char *v = (char *)g.dev;
  g.d_nc = (int64_t *)v;
  g.d_step = (int64_t *)(v + 8);
  g.d_cnt = (int64_t *)(v + 16);
  g.d_ovf = (int *)(v + 32);
  g.d_snap = (int *)(v + 36);
  g.d_bp = (int64_t *)(v + 40);
  g.d_pend = (int64_t *)(v + 48);  // 3 counters of the step in flight
  g.d_log = (int64_t *)(v + 256);
  if ((e = cudaMemset(g.dev, 0, 256)) != cudaSuccess) return cuda_error(e, "graph memset");
  if ((e = block_sort_prepare()) != cudaSuccess) return cuda_error(e, "pair sort attributes");
  if ((e = forces_fixed_init(s->ctx->stream, g.fs, contact_cap, n)) != cudaSuccess) return cuda_error(e, "forces init");
  delta_status ds = detect_fixed_init(s->ctx->stream, g.ds, pair_cap, contact_cap);
  if (ds != DELTA_OK) return ds;
  if (s->plan.skin > 0.0) {
    // the skin list, sized from the pairs within reach + skin now (half again, and more)
    int64_t found = 0;
    if ((ds = skin_count(s->ctx->stream, s->scene, s->plan, g.bp, g.temp, g.temp_bytes, &found)) != DELTA_OK)
      return ds;
    const int64_t cap = std::max<int64_t>(1024, found + found / 2 + 1024);
    const size_t tb = skin_temp_bytes(s->scene, s->plan, cap) + 256;
    if (tb > g.temp_bytes) {
      cudaFree(g.temp);
      g.temp = nullptr;
      if ((e = cudaMalloc(&g.temp, tb)) != cudaSuccess) return cuda_error(e, "skin temp");
      g.temp_bytes = tb;
    }
    if ((e = cudaMalloc(&g.sk, skin_bytes(n, cap))) != cudaSuccess) return cuda_error(e, "skin list");
    g.skin = carve_skin(g.sk, n, cap);
    if ((e = cudaMemset(g.sk, 0, 256)) != cudaSuccess || (e = cudaMemset(g.skin.need, 0xff, sizeof(int))) != cudaSuccess)
      return cuda_error(e, "skin init");
  }
  if ((e = cudaStreamSynchronize(s->ctx->stream)) != cudaSuccess) return cuda_error(e, "graph init");
  return DELTA_OK;
}

// The step's broadphase from the skin list, under capture on g.stream: the check sets
// the condition of an IF node whose body (captured from stream2) rebuilds the list; the
// filter then forms the step's pairs.  k counts the kernels of every step; the body's
// kernels go to g.rebuild_kernels.
static delta_status graph_skin_broadphase(delta_sim *s, int &k) {
  delta_sim::Graph &g = s->g;
  cudaStream_t st = g.stream;
  cudaError_t e;
  if (!g.stream2 && (e = cudaStreamCreateWithFlags(&g.stream2, cudaStreamNonBlocking)) != cudaSuccess)
    return cuda_error(e, "skin stream");
  cudaStreamCaptureStatus cs;
  cudaGraph_t cg = nullptr;
  if ((e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, nullptr, nullptr)) != cudaSuccess)
    return cuda_error(e, "skin capture info");
  cudaGraphConditionalHandle h;
  if ((e = cudaGraphConditionalHandleCreate(&h, cg, 0, 0)) != cudaSuccess) return cuda_error(e, "skin condition");
  if ((e = skin_check(st, s->scene, s->plan, g.skin, h, k)) != cudaSuccess) return cuda_error(e, "skin check");
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  if ((e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, &deps, &nd)) != cudaSuccess)
    return cuda_error(e, "skin capture info");
  cudaGraphNodeParams np{};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeIf;
  np.conditional.size = 1;
  cudaGraphNode_t cn;
  if ((e = cudaGraphAddNode(&cn, cg, deps, nd, &np)) != cudaSuccess) return cuda_error(e, "skin conditional node");
  if ((e = cudaStreamUpdateCaptureDependencies(st, &cn, 1, cudaStreamSetCaptureDependencies)) != cudaSuccess)
    return cuda_error(e, "skin capture dependencies");
  cudaGraph_t body = np.conditional.phGraph_out[0];
  if ((e = cudaStreamBeginCaptureToGraph(g.stream2, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
      cudaSuccess)
    return cuda_error(e, "skin body capture");
  int rk = 0;
  const cudaError_t eb = skin_build(g.stream2, s->scene, s->plan, g.skin, g.bp, g.temp, g.temp_bytes, g.d_ovf, rk);
  cudaGraph_t out = nullptr;
  e = cudaStreamEndCapture(g.stream2, &out);
  if (eb != cudaSuccess) return cuda_error(eb, "skin build");
  if (e != cudaSuccess) return cuda_error(e, "skin body capture");
  g.rebuild_kernels = rk;
  if ((e = skin_filter(st, s->scene, s->plan, g.skin, g.pa, g.pb, g.pair_cap, g.d_ovf, g.d_pend, g.bp, g.temp,
                       g.temp_bytes, k)) != cudaSuccess)
    return cuda_error(e, "skin filter");
  return DELTA_OK;
}

// The skin list's rebuilds inside the graph since the last count: their kernels go to the
// context's launch count, the builds to the simulation's total.
static delta_status graph_count_rebuilds(delta_sim *s) {
  delta_sim::Graph &g = s->g;
  if (g.skin.cap <= 0) return DELTA_OK;
  unsigned long long rb = 0;
  cudaError_t e = cudaMemcpy(&rb, g.skin.rebuilds, 8, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_error(e, "skin rebuilds");
  s->ctx->launches += (int64_t)(rb - g.rebuilds_seen) * g.rebuild_kernels;
  s->skin_rebuilds += (int64_t)(rb - g.rebuilds_seen);
  g.rebuilds_seen = rb;
  return DELTA_OK;
}

// Enqueues one fixed-capacity step on g.stream (used under capture).
static delta_status graph_enqueue_step(delta_sim *s, const delta_step_params &p) {
  delta_sim::Graph &g = s->g;
  cudaStream_t st = g.stream;
  int k = 0;
  delta_status ds = forces_run_fixed(st, s->scene, g.c, g.d_nc, p, s->F, s->T, s->has, g.fs, g.temp, g.temp_bytes, k);
  if (ds != DELTA_OK) return ds;
  cudaError_t le = launch_dep(true, k_bodies, blocks_for(s->scene.n_bodies, 128), 128, 0, st, s->scene, p, s->F, s->T,
                              s->has, g.d_ovf, g.d_snap, s->epoch);
  if (le != cudaSuccess) return cuda_error(le, "body update");
  if (g.skin.cap > 0) {
    if ((ds = graph_skin_broadphase(s, k)) != DELTA_OK) return ds;
  } else if ((ds = broadphase_run_fixed(st, s->scene, s->plan, g.pa, g.pb, g.pair_cap, g.d_ovf, g.d_pend, g.bp,
                                        g.temp, g.temp_bytes, k)) != DELTA_OK) {
    return ds;
  }
  // vertices of the bodies the narrowphase reads this step: formed from the poses by the
  // certified driver, updated here for the others
  const bool posed = s->driver == DELTA_DRV_BF_CERT || s->driver == DELTA_DRV_BF_CULLED || s->driver == DELTA_DRV_LEARNED;
  const Pose pose = sim_pose(s);
  if (!posed) {
    cudaError_t ve = launch_dep(true, k_mark_pair_bodies, blocks_for(g.pair_cap), 256, 0, st, g.pa, g.pb, g.pair_cap,
                                s->epoch, s->stamp);
    if (ve == cudaSuccess)
      ve = launch_dep(true, k_vertices, vertex_blocks(s->scene.n_bodies), 256, 0, st, s->scene, g.d_ovf, nullptr,
                      s->stamp, s->epoch);
    if (ve != cudaSuccess) return cuda_error(ve, "step vertices");
    k += 2;
  }
  delta_meshes m{s->scene.n_bodies, s->scene.tri_offset, s->scene.x, s->scene.y, s->scene.z,
                 s->scene.eps,      s->scene.friction,   s->ids};
  const int64_t before = s->ctx->launches;
  if ((ds = detect_run_fixed(s->ctx, st, s->driver, m, g.pa, g.pb, g.pair_cap, g.c, g.d_nc, g.d_ovf, 1, g.d_pend + 1,
                             nullptr, g.ds, g.temp, g.temp_bytes, posed ? &pose : nullptr, s->tri_bits)) != DELTA_OK)
    return ds;
  k += (int)(s->ctx->launches - before);
  s->ctx->launches = before;
  const cudaError_t ee = launch_dep(true, k_step_end, 1, 1, 0, st, g.d_snap, g.d_ovf, g.d_nc, g.d_log, g.log_len,
                                    g.d_step, g.d_pend, g.d_bp, g.d_cnt);
  if (ee != cudaSuccess) return cuda_error(ee, "step end");
  g.kernels = k + 2;
  return cuda_error(cudaGetLastError(), "graph step");
}

static delta_status graph_capture(delta_sim *s, const delta_step_params &p) {
  delta_sim::Graph &g = s->g;
  if (g.exec) cudaGraphExecDestroy(g.exec);
  if (g.graph) cudaGraphDestroy(g.graph);
  g.exec = nullptr;
  g.graph = nullptr;
  cudaError_t e = cudaStreamBeginCapture(g.stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return cuda_error(e, "begin capture");
  delta_status ds = graph_enqueue_step(s, p);
  cudaGraph_t graph = nullptr;
  e = cudaStreamEndCapture(g.stream, &graph);
  if (ds != DELTA_OK) {
    if (graph) cudaGraphDestroy(graph);
    return ds;
  }
  if (e != cudaSuccess) return cuda_error(e, "end capture");
  g.graph = graph;
  if ((e = cudaGraphInstantiate(&g.exec, g.graph, 0)) != cudaSuccess) return cuda_error(e, "graph instantiate");
  g.params = p;
  g.launch_epoch = s->ctx->launch_epoch;
  g.captured = true;
  return DELTA_OK;
}

// Host contact list (sim->c) <-> graph contact buffer.
static delta_status copy_contacts(const delta_contacts &src, const delta_contacts &dst, int64_t n, cudaStream_t st) {
  cudaError_t e = cudaSuccess;
  const int64_t ic = src.capacity, oc = dst.capacity;
  for (int k = 0; k < 3 && e == cudaSuccess; ++k) {
    e = cudaMemcpyAsync(dst.x + k * oc, src.x + k * ic, 8 * n, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dst.normal + k * oc, src.normal + k * ic, 8 * n, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dst.P + k * oc, src.P + k * ic, 8 * n, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dst.Q + k * oc, src.Q + k * ic, 8 * n, cudaMemcpyDeviceToDevice, st);
  }
  const void *srcs[] = {src.depth, src.eps_total, src.master, src.slave, src.tri_a, src.tri_b, src.penetration,
                        src.friction};
  void *dsts[] = {dst.depth, dst.eps_total, dst.master, dst.slave, dst.tri_a, dst.tri_b, dst.penetration,
                  dst.friction};
  const size_t sz[] = {8, 8, 4, 4, 4, 4, 4, 1};
  for (int k = 0; k < 8 && e == cudaSuccess; ++k)
    e = cudaMemcpyAsync(dsts[k], srcs[k], sz[k] * n, cudaMemcpyDeviceToDevice, st);
  return cuda_error(e, "copy contacts");
}

}  // namespace delta

using namespace delta;

extern "C" {

delta_status delta_forces(delta_ctx *ctx, const delta_scene *scene, const delta_contacts *contacts,
                          int64_t n_contacts, const delta_step_params *params, double *force, double *torque,
                          uint8_t *has_contact) {
  if (!ctx || !scene || !params || !force || !torque || !has_contact || (n_contacts > 0 && !contacts))
    return set_error(DELTA_ERR_INVALID, "delta_forces: null argument");
  if (n_contacts < 0 || (contacts && n_contacts > contacts->capacity))
    return set_error(DELTA_ERR_INVALID, "delta_forces: bad contact count");
  delta_contacts empty{};
  return forces_run(ctx, *scene, contacts ? *contacts : empty, n_contacts, *params, force, torque, has_contact);
}

delta_status delta_contact_forces(delta_ctx *ctx, int64_t n_groups, const int64_t *offset,
                                  const delta_contacts *contacts, const double *pos_a, const double *ang_a,
                                  const double *lin_a, const double *mass_a, const double *pos_b,
                                  const double *ang_b, const double *lin_b, const double *mass_b,
                                  const delta_step_params *params, double *force, double *torque) {
  if (!ctx || !params) return set_error(DELTA_ERR_INVALID, "delta_contact_forces: null argument");
  if (n_groups < 0) return set_error(DELTA_ERR_INVALID, "delta_contact_forces: negative size");
  if (n_groups == 0) return DELTA_OK;
  if (!offset || !contacts || !pos_a || !ang_a || !lin_a || !mass_a || !pos_b || !ang_b || !lin_b || !mass_b ||
      !force || !torque || (contacts->capacity > 0 && (!contacts->x || !contacts->normal || !contacts->depth ||
                                                       !contacts->friction)))
    return set_error(DELTA_ERR_INVALID, "delta_contact_forces: null argument");
  ContactView cv{contacts->x, contacts->normal, contacts->depth, contacts->master, contacts->slave,
                 contacts->friction, contacts->capacity};
  GroupKin g{pos_a, ang_a, lin_a, mass_a, pos_b, ang_b, lin_b, mass_b};
  k_contact_forces_groups<<<(unsigned)((n_groups + 127) / 128), 128, 0, ctx->stream>>>(n_groups, offset, cv, g,
                                                                                      *params, force, torque);
  ctx->launches += 1;
  return cuda_error(cudaGetLastError(), "delta_contact_forces launch");
}

delta_status delta_update_angular(delta_ctx *ctx, int32_t n, double *ref_ang, const double *rot,
                                  const double *inertia, const double *inverse, const double *torque, double step) {
  if (!ctx || n < 0) return set_error(DELTA_ERR_INVALID, "delta_update_angular: bad argument");
  if (n == 0) return DELTA_OK;
  if (!ref_ang || !rot || !inertia || !inverse || !torque)
    return set_error(DELTA_ERR_INVALID, "delta_update_angular: null argument");
  delta_scene s{};
  s.n_bodies = n;
  s.ref_ang = ref_ang;
  s.rot = const_cast<double *>(rot);
  s.inertia = inertia;
  s.inverse = inverse;
  k_update_angular_only<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(s, torque, step);
  ctx->launches += 1;
  return cuda_error(cudaGetLastError(), "delta_update_angular launch");
}

delta_status delta_update_rotation(delta_ctx *ctx, int32_t n, double *ang, const double *ref_ang, double *rot,
                                   double step) {
  if (!ctx || n < 0) return set_error(DELTA_ERR_INVALID, "delta_update_rotation: bad argument");
  if (n == 0) return DELTA_OK;
  if (!ang || !ref_ang || !rot) return set_error(DELTA_ERR_INVALID, "delta_update_rotation: null argument");
  delta_scene s{};
  s.n_bodies = n;
  s.ang = ang;
  s.ref_ang = const_cast<double *>(ref_ang);
  s.rot = rot;
  k_update_rotation_only<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(s, step);
  ctx->launches += 1;
  return cuda_error(cudaGetLastError(), "delta_update_rotation launch");
}

delta_status delta_update_vertices(delta_ctx *ctx, int64_t n_vertices, const int32_t *body, int32_t n_bodies,
                                   double *x, double *y, double *z, const double *rx, const double *ry,
                                   const double *rz, const double *rot, const double *pos, const double *ref_pos) {
  if (!ctx || n_vertices < 0 || n_bodies < 0) return set_error(DELTA_ERR_INVALID, "delta_update_vertices: bad size");
  if (n_vertices == 0) return DELTA_OK;
  if (n_bodies == 0 || !x || !y || !z || !rx || !ry || !rz || !rot || !pos || !ref_pos || (!body && n_bodies != 1))
    return set_error(DELTA_ERR_INVALID, "delta_update_vertices: null argument");
  k_update_vertices_only<<<(unsigned)((n_vertices + 127) / 128), 128, 0, ctx->stream>>>(
      n_vertices, body, n_bodies, x, y, z, rx, ry, rz, rot, pos, ref_pos);
  ctx->launches += 1;
  return cuda_error(cudaGetLastError(), "delta_update_vertices launch");
}

delta_status delta_integrate(delta_ctx *ctx, const delta_scene *scene, const delta_step_params *params,
                             const double *force, const double *torque, const uint8_t *has_contact) {
  if (!ctx || !scene || !params || !force || !torque || !has_contact)
    return set_error(DELTA_ERR_INVALID, "delta_integrate: null argument");
  int64_t ntri = 0;
  cudaError_t e = cudaMemcpyAsync(&ntri, scene->tri_offset + scene->n_bodies, sizeof(int64_t),
                                  cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_error(e, "delta_integrate");
  return integrate_run(ctx, *scene, *params, force, torque, has_contact, 3 * ntri);
}

delta_status delta_broadphase(delta_ctx *ctx, const delta_scene *scene, int32_t *pair_a, int32_t *pair_b,
                              int64_t capacity, int64_t *n_out) {
  if (!ctx || !scene || !n_out || (capacity > 0 && (!pair_a || !pair_b)))
    return set_error(DELTA_ERR_INVALID, "delta_broadphase: null argument");
  BroadphasePlan plan;
  delta_status ds = broadphase_plan(ctx, *scene, plan);
  if (ds == DELTA_OK) ds = broadphase_run(ctx, *scene, plan, pair_a, pair_b, capacity, n_out);
  cudaStreamSynchronize(ctx->stream);
  plan.release();
  return ds;
}

delta_status delta_sim_create(delta_ctx *ctx, const delta_scene *scene, int driver, delta_sim **out) {
  if (!ctx || !scene || !out) return set_error(DELTA_ERR_INVALID, "delta_sim_create: null argument");
  if (driver != DELTA_DRV_BF && driver != DELTA_DRV_BF_CERT && driver != DELTA_DRV_BF_CULLED &&
      driver != DELTA_DRV_LEARNED)
    return set_error(DELTA_ERR_UNSUPPORTED, "delta_sim_create: the time step runs DELTA_DRV_BF, DELTA_DRV_BF_CERT, "
                                            "DELTA_DRV_BF_CULLED or DELTA_DRV_LEARNED");
  delta_sim *s = new delta_sim();
  s->ctx = ctx;
  s->scene = *scene;
  s->driver = driver;
  const int32_t n = scene->n_bodies;
  std::vector<int64_t> off((size_t)n + 1);
  cudaError_t e = cudaMemcpy(off.data(), scene->tri_offset, sizeof(int64_t) * ((size_t)n + 1), cudaMemcpyDeviceToHost);
  delta_status ds = DELTA_OK;
  if (e != cudaSuccess) ds = cuda_error(e, "sim create");
  s->n_tri = off[n];
  int64_t max_tri = 1;
  for (int32_t i = 0; i < n; ++i) max_tri = std::max<int64_t>(max_tri, off[i + 1] - off[i]);
  s->tri_bits = max_tri <= 65536 ? bits_for(max_tri - 1) : 16;
  if (ds == DELTA_OK && (e = cudaMalloc(&s->ids, sizeof(int32_t) * n)) != cudaSuccess) ds = cuda_error(e, "ids");
  if (ds == DELTA_OK && ((e = cudaMalloc(&s->stamp, sizeof(uint32_t) * ((size_t)n + 1))) != cudaSuccess ||
                         (e = cudaMemset(s->stamp, 0, sizeof(uint32_t) * ((size_t)n + 1))) != cudaSuccess))
    ds = cuda_error(e, "vertex stamps");
  if (ds == DELTA_OK) s->epoch = s->stamp + n;
  if (ds == DELTA_OK && (e = cudaMalloc(&s->reach, 56 * (size_t)n + 64)) != cudaSuccess) ds = cuda_error(e, "reach");
  if (ds == DELTA_OK) {
    s->obox = s->reach + n;
    k_reach_boxes<<<vertex_blocks(n), 256, 0, ctx->stream>>>(*scene, s->reach, s->obox);
    ctx->launches += 1;
  }
  if (ds == DELTA_OK && (e = cudaMalloc(&s->F, sizeof(double) * 6 * n + n)) != cudaSuccess) ds = cuda_error(e, "F");
  if (ds == DELTA_OK) {
    s->T = s->F + 3 * n;
    s->has = (uint8_t *)(s->T + 3 * n);
    k_iota32<<<blocks_for(n), 256, 0, ctx->stream>>>(s->ids, n);
    ctx->launches += 1;
    ds = broadphase_plan(ctx, *scene, s->plan);
  }
  if (ds == DELTA_OK) ds = alloc_contacts(s, 1 << 16);
  if (ds == DELTA_OK) ds = alloc_pairs(s, 1 << 14);
  if (ds != DELTA_OK) {
    delta_sim_destroy(s);
    return ds;
  }
  *out = s;
  return DELTA_OK;
}

delta_status delta_sim_step(delta_sim *s, const delta_step_params *params, int32_t nsteps,
                            int64_t *contacts_per_step) {
  if (!s || !params || nsteps < 0) return set_error(DELTA_ERR_INVALID, "delta_sim_step: bad argument");
  for (int32_t k = 0; k < nsteps; ++k) {
    delta_status ds = forces_run(s->ctx, s->scene, s->c, s->n_contacts, *params, s->F, s->T, s->has);
    if (ds != DELTA_OK) return ds;
    k_bodies<<<blocks_for(s->scene.n_bodies, 128), 128, 0, s->ctx->stream>>>(s->scene, *params, s->F, s->T, s->has,
                                                                              nullptr, nullptr, nullptr);
    s->ctx->launches += 1;
    if ((ds = sim_detect(s)) != DELTA_OK) return ds;
    s->counters[0] += 1;
    if (contacts_per_step) contacts_per_step[k] = s->n_contacts;
  }
  return sim_all_vertices(s, s->ctx->stream);
}

delta_status delta_sim_autotune(delta_sim *s, int32_t reps, int32_t *choice, float *ms_out) {
  if (!s || reps < 1 || !choice) return set_error(DELTA_ERR_INVALID, "delta_sim_autotune: bad argument");
  delta_ctx *ctx = s->ctx;
  if (s->driver != DELTA_DRV_BF_CERT && s->driver != DELTA_DRV_BF_CULLED && s->driver != DELTA_DRV_LEARNED) {
    choice[0] = choice[1] = 0;  // nothing to tune: the pair kernels take delta_set_pair_launch
    if (ms_out) *ms_out = 0.f;
    return DELTA_OK;
  }
  int cull_max = 0, surv_max = 0;
  cudaError_t e = detect_launch_limits(s->driver, &cull_max, &surv_max);
  if (e != cudaSuccess) return cuda_error(e, "delta_sim_autotune: occupancy");
  // one detection of the current state (grows the pair and contact buffers to fit), then
  // every launch shape on the same pairs; detection changes no state but the contacts,
  // which each run writes alike
  const int64_t saved[4] = {s->counters[0], s->counters[1], s->counters[2], s->counters[3]};
  const int saved_shape[2] = {ctx->cull_blocks_per_sm, ctx->surv_blocks_per_sm};
  delta_status ds = sim_detect(s);
  std::copy(saved, saved + 4, s->counters);
  if (ds != DELTA_OK) return ds;
  std::vector<int> cull_c, surv_c;
  for (int c = 1; c <= cull_max; c = c < 2 ? c + 1 : c + 2) cull_c.push_back(c);
  for (int c = 1; c <= surv_max; ++c) surv_c.push_back(c);
  if (cull_c.empty()) cull_c.push_back(0);
  if (surv_c.empty()) surv_c.push_back(0);
  const Pose pose = sim_pose(s);
  delta_meshes m{s->scene.n_bodies, s->scene.tri_offset, s->scene.x, s->scene.y, s->scene.z,
                 s->scene.eps,      s->scene.friction,   s->ids};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  if ((e = cudaEventCreate(&ev[0])) != cudaSuccess || (e = cudaEventCreate(&ev[1])) != cudaSuccess) {
    for (cudaEvent_t x : ev)
      if (x) cudaEventDestroy(x);
    return cuda_error(e, "delta_sim_autotune: events");
  }
  float best = -1.f;
  int best_c = 0, best_s = 0;
  for (int cc : cull_c) {
    for (int sc : surv_c) {
      ctx->cull_blocks_per_sm = cc;
      ctx->surv_blocks_per_sm = sc;
      std::vector<float> t;
      for (int r = 0; r <= reps && ds == DELTA_OK; ++r) {  // r == 0: warm-up
        int64_t nc = 0;
        if ((e = cudaEventRecord(ev[0], ctx->stream)) != cudaSuccess) break;
        if (s->last_pairs > 0)
          ds = detect_run(ctx, s->driver, DELTA_F64, m, s->pa, s->pb, s->last_pairs, &s->c, &nc, nullptr, nullptr,
                          &pose);
        if (ds != DELTA_OK) break;
        if ((e = cudaEventRecord(ev[1], ctx->stream)) != cudaSuccess || (e = cudaEventSynchronize(ev[1])) != cudaSuccess)
          break;
        float ms = 0.f;
        if ((e = cudaEventElapsedTime(&ms, ev[0], ev[1])) != cudaSuccess) break;
        if (r > 0) t.push_back(ms);
      }
      if (ds != DELTA_OK || e != cudaSuccess) break;
      std::sort(t.begin(), t.end());
      const float med = t[t.size() / 2];
      if (best < 0.f || med < best) {
        best = med;
        best_c = cc;
        best_s = sc;
      }
    }
    if (ds != DELTA_OK || e != cudaSuccess) break;
  }
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  if (ds == DELTA_OK && e != cudaSuccess) ds = cuda_error(e, "delta_sim_autotune");
  if (ds != DELTA_OK) {
    ctx->cull_blocks_per_sm = saved_shape[0];
    ctx->surv_blocks_per_sm = saved_shape[1];
    ctx->launch_epoch += 1;
    return ds;
  }
  ctx->cull_blocks_per_sm = choice[0] = best_c;
  ctx->surv_blocks_per_sm = choice[1] = best_s;
  ctx->launch_epoch += 1;  // recorded steps hold the old launch shapes
  if (ms_out) *ms_out = best;
  return DELTA_OK;
}

delta_status delta_sim_contacts(delta_sim *s, const delta_contacts *out, int64_t *n_out) {
  if (!s || !out || !n_out) return set_error(DELTA_ERR_INVALID, "delta_sim_contacts: null argument");
  *n_out = s->n_contacts;
  const int64_t n = s->n_contacts < out->capacity ? s->n_contacts : out->capacity;
  cudaStream_t st = s->ctx->stream;
  const int64_t ic = s->c.capacity, oc = out->capacity;
  cudaError_t e = cudaSuccess;
  if (n > 0) {
    auto cp3 = [&](double *dst, const double *src) {
      for (int k = 0; k < 3 && e == cudaSuccess; ++k)
        e = cudaMemcpyAsync(dst + k * oc, src + k * ic, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
    };
    cp3(out->x, s->c.x);
    cp3(out->normal, s->c.normal);
    cp3(out->P, s->c.P);
    cp3(out->Q, s->c.Q);
    const void *srcs[] = {s->c.depth, s->c.eps_total, s->c.master, s->c.slave, s->c.tri_a, s->c.tri_b,
                          s->c.penetration, s->c.friction};
    void *dsts[] = {out->depth, out->eps_total, out->master, out->slave, out->tri_a, out->tri_b, out->penetration,
                    out->friction};
    const size_t sz[] = {8, 8, 4, 4, 4, 4, 4, 1};
    for (int k = 0; k < 8 && e == cudaSuccess; ++k)
      e = cudaMemcpyAsync(dsts[k], srcs[k], sz[k] * n, cudaMemcpyDeviceToDevice, st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_error(e, "delta_sim_contacts");
  if (s->n_contacts > out->capacity) return set_error(DELTA_ERR_CAPACITY, "delta_sim_contacts: capacity");
  return DELTA_OK;
}

delta_status delta_sim_step_graph(delta_sim *s, const delta_step_params *params, int32_t nsteps,
                                  int64_t *contacts_per_step) {
  if (!s || !params || nsteps < 0) return set_error(DELTA_ERR_INVALID, "delta_sim_step_graph: bad argument");
  if (nsteps == 0) return DELTA_OK;
  delta_sim::Graph &g = s->g;
  cudaError_t e;
  delta_status ds;
  if (!g.stream) {
    if ((e = cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&g.ev, cudaEventDisableTiming)) != cudaSuccess)
      return cuda_error(e, "graph stream");
  }
  int32_t done = 0;
  if (s->counters[0] == 0) {  // observe one detection before sizing the fixed buffers
    if ((ds = delta_sim_step(s, params, 1, contacts_per_step)) != DELTA_OK) return ds;
    done = 1;
  }
  const bool requested = s->graph_pair_cap > 0 || s->graph_contact_cap > 0;
  int64_t want_pairs = std::max<int64_t>(1024, 2 * std::max<int64_t>(s->counters[1] / std::max<int64_t>(1, s->counters[0]), 1));
  int64_t want_contacts = std::max<int64_t>(2048, 4 * s->n_contacts);
  if (s->graph_pair_cap > 0) want_pairs = s->graph_pair_cap;
  if (s->graph_contact_cap > 0) want_contacts = s->graph_contact_cap;
  want_contacts = std::max<int64_t>(want_contacts, s->n_contacts);  // the current list must fit
  s->graph_pair_cap = s->graph_contact_cap = 0;
  // The buffers (and the recorded graph) are kept from call to call while the current
  // contacts and the step log fit; a replay that overflows grows them.  They are sized anew
  // on the first call, on a capacity request, or when the contacts or the log outgrew them.
  if (!g.pa || requested || g.contact_cap < s->n_contacts || g.log_len < nsteps) {
    const bool fresh = !g.pa || requested;
    if ((ds = graph_alloc(s, fresh ? want_pairs : std::max(g.pair_cap, want_pairs),
                          fresh ? want_contacts : std::max(g.contact_cap, want_contacts),
                          std::max<int64_t>({g.log_len, (int64_t)nsteps, 4096}))) != DELTA_OK)
      return ds;
  }
  if (memcmp(&g.params, params, sizeof(*params)) != 0 || g.launch_epoch != s->ctx->launch_epoch) g.captured = false;
  // hand the current contacts to the graph buffers; ctx stream work must be done first
  if ((e = cudaEventRecord(g.ev, s->ctx->stream)) != cudaSuccess ||
      (e = cudaStreamWaitEvent(g.stream, g.ev, 0)) != cudaSuccess)
    return cuda_error(e, "graph order");
  if ((ds = copy_contacts(s->c, g.c, s->n_contacts, g.stream)) != DELTA_OK) return ds;
  int64_t hv[2] = {s->n_contacts, 0};
  if ((e = cudaMemcpyAsync(g.d_nc, &hv[0], 8, cudaMemcpyHostToDevice, g.stream)) != cudaSuccess ||
      (e = cudaMemsetAsync(g.d_step, 0, 8, g.stream)) != cudaSuccess ||
      (e = cudaMemsetAsync(g.d_cnt, 0, 16, g.stream)) != cudaSuccess ||
      (e = cudaMemsetAsync(g.d_bp, 0, 8, g.stream)) != cudaSuccess ||
      (e = cudaMemsetAsync(g.d_pend, 0, 24, g.stream)) != cudaSuccess ||
      (e = cudaMemsetAsync(g.d_ovf, 0, 8, g.stream)) != cudaSuccess ||
      (g.skin.cap > 0 && (e = cudaMemsetAsync(g.skin.need, 0xff, sizeof(int), g.stream)) != cudaSuccess) ||
      (e = cudaStreamSynchronize(g.stream)) != cudaSuccess)
    return cuda_error(e, "graph setup");
  int32_t base = done;  // steps completed before the current batch of launches
  while (done < nsteps) {
    if (!g.captured && (ds = graph_capture(s, *params)) != DELTA_OK) return ds;
    const int32_t batch = nsteps - done;
    for (int32_t k = 0; k < batch; ++k)
      if ((e = cudaGraphLaunch(g.exec, g.stream)) != cudaSuccess) return cuda_error(e, "graph launch");
    s->ctx->launches += (int64_t)g.kernels * batch;
    int64_t dev_step = 0;
    int ovf = 0;
    if ((e = cudaMemcpyAsync(&dev_step, g.d_step, 8, cudaMemcpyDeviceToHost, g.stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&ovf, g.d_ovf, 4, cudaMemcpyDeviceToHost, g.stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(g.stream)) != cudaSuccess)
      return cuda_error(e, "graph sync");
    // dev_step counts graph steps (since setup) whose integration ran
    if (contacts_per_step) {
      const int64_t first = done - base;
      const int64_t n = dev_step - first;
      if (n > 0 && (e = cudaMemcpy(contacts_per_step + done, g.d_log + first, 8 * n, cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_error(e, "graph log");
    }
    s->counters[0] += dev_step - (done - base);
    done = base + (int32_t)dev_step;
    if (!ovf) break;
    // overflow in the detection of the last integrated step: grow, detect again, recapture
    unsigned long long pc = 0;
    if ((e = cudaMemcpy(&pc, broadphase_fixed_count(g.bp, s->scene.n_bodies), 8, cudaMemcpyDeviceToHost)) !=
        cudaSuccess)
      return cuda_error(e, "overflow counts");
    if ((e = cudaStreamSynchronize(s->ctx->stream)) != cudaSuccess) return cuda_error(e, "sync");
    if ((ds = sim_detect(s)) != DELTA_OK) return ds;  // non-graph detection of the current state
    if (contacts_per_step && done > 0) contacts_per_step[done - 1] = s->n_contacts;
    int64_t saved_log = g.log_len, seg_cnt[2] = {0, 0}, seg_bp = 0;
    if ((e = cudaMemcpy(seg_cnt, g.d_cnt, 16, cudaMemcpyDeviceToHost)) != cudaSuccess ||
        (e = cudaMemcpy(&seg_bp, g.d_bp, 8, cudaMemcpyDeviceToHost)) != cudaSuccess)
      return cuda_error(e, "counters");
    s->counters[1] += seg_bp;
    s->counters[2] += seg_cnt[0];
    s->counters[3] += seg_cnt[1];
    if ((ds = graph_count_rebuilds(s)) != DELTA_OK) return ds;
    if ((ds = graph_alloc(s, std::max<int64_t>(2 * g.pair_cap, 2 * (int64_t)pc), std::max<int64_t>(2 * g.contact_cap,
                          4 * s->n_contacts), saved_log)) != DELTA_OK)
      return ds;
    if ((ds = copy_contacts(s->c, g.c, s->n_contacts, g.stream)) != DELTA_OK) return ds;
    hv[0] = s->n_contacts;
    if ((e = cudaMemcpyAsync(g.d_nc, &hv[0], 8, cudaMemcpyHostToDevice, g.stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(g.stream)) != cudaSuccess)
      return cuda_error(e, "graph restart");
    base = done;
  }
  // counters and contacts back to the simulation object
  int64_t cnt[2] = {0, 0}, nc = 0, bp = 0;
  if ((e = cudaMemcpy(cnt, g.d_cnt, 16, cudaMemcpyDeviceToHost)) != cudaSuccess ||
      (e = cudaMemcpy(&bp, g.d_bp, 8, cudaMemcpyDeviceToHost)) != cudaSuccess ||
      (e = cudaMemcpy(&nc, g.d_nc, 8, cudaMemcpyDeviceToHost)) != cudaSuccess)
    return cuda_error(e, "graph counters");
  s->counters[1] += bp;
  s->counters[2] += cnt[0];
  s->counters[3] += cnt[1];
  if ((ds = graph_count_rebuilds(s)) != DELTA_OK) return ds;
  if (nc > s->c.capacity && (ds = alloc_contacts(s, nc + nc / 2 + 1024)) != DELTA_OK) return ds;
  if ((ds = copy_contacts(g.c, s->c, nc, g.stream)) != DELTA_OK) return ds;
  if ((ds = sim_all_vertices(s, g.stream)) != DELTA_OK) return ds;
  if ((e = cudaStreamSynchronize(g.stream)) != cudaSuccess) return cuda_error(e, "graph end");
  s->n_contacts = nc;
  return DELTA_OK;
}

delta_status delta_sim_skin_stats(delta_sim *s, double *skin, int64_t *capacity, int64_t *rebuilds) {
  if (!s || !skin || !capacity || !rebuilds) return set_error(DELTA_ERR_INVALID, "delta_sim_skin_stats: bad argument");
  *skin = s->plan.skin;
  *capacity = s->g.skin.cap;
  *rebuilds = s->skin_rebuilds;
  return DELTA_OK;
}

delta_status delta_sim_set_graph_capacity(delta_sim *s, int64_t pair_capacity, int64_t contact_capacity) {
  if (!s || pair_capacity < 1 || contact_capacity < 1)
    return set_error(DELTA_ERR_INVALID, "delta_sim_set_graph_capacity: bad argument");
  s->graph_pair_cap = pair_capacity;
  s->graph_contact_cap = contact_capacity;
  return DELTA_OK;
}

delta_status delta_sim_counters(const delta_sim *s, int64_t out[4]) {
  if (!s || !out) return set_error(DELTA_ERR_INVALID, "delta_sim_counters: null argument");
  for (int k = 0; k < 4; ++k) out[k] = s->counters[k];
  return DELTA_OK;
}

delta_status delta_sim_destroy(delta_sim *s) {
  if (!s) return DELTA_OK;
  cudaStreamSynchronize(s->ctx->stream);
  if (s->g.stream) cudaStreamSynchronize(s->g.stream);
  graph_release(s->g);
  if (s->g.ev) cudaEventDestroy(s->g.ev);
  if (s->g.stream) cudaStreamDestroy(s->g.stream);
  if (s->g.stream2) cudaStreamDestroy(s->g.stream2);
  s->plan.release();
  if (s->ids) cudaFree(s->ids);
  if (s->stamp) cudaFree(s->stamp);
  if (s->reach) cudaFree(s->reach);
  if (s->F) cudaFree(s->F);
  if (s->c_mem) cudaFree(s->c_mem);
  if (s->pa) cudaFree(s->pa);
  delete s;
  return DELTA_OK;
}

delta_status delta_sim_write_vtk(delta_sim *sim, const char *path, int32_t step) {
  if (!sim || !path) return set_error(DELTA_ERR_INVALID, "delta_sim_write_vtk: bad argument");
  // the vertices after the last step (graph replays run on the simulation's own stream)
  if (sim->g.stream) {
    const cudaError_t e = cudaStreamSynchronize(sim->g.stream);
    if (e != cudaSuccess) return cuda_error(e, "delta_sim_write_vtk: graph stream");
  }
  delta_meshes m{sim->scene.n_bodies, sim->scene.tri_offset, sim->scene.x, sim->scene.y, sim->scene.z,
                 sim->scene.eps, sim->scene.friction, sim->ids};
  return delta_write_vtk(sim->ctx, path, step, &m);
}

delta_status delta_sim_write_vtu(delta_sim *sim, const char *path, int32_t step) {
  if (!sim || !path) return set_error(DELTA_ERR_INVALID, "delta_sim_write_vtu: bad argument");
  cudaError_t e = cudaSuccess;
  if (sim->g.stream) e = cudaStreamSynchronize(sim->g.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(sim->ctx->stream);
  if (e != cudaSuccess) return cuda_error(e, "delta_sim_write_vtu: sync");
  const int64_t n = sim->scene.n_bodies;
  std::vector<double> pos(3 * n), vel(3 * n), eps(n);
  if ((e = cudaMemcpy(pos.data(), sim->scene.pos, 8 * 3 * n, cudaMemcpyDeviceToHost)) == cudaSuccess &&
      (e = cudaMemcpy(vel.data(), sim->scene.vel, 8 * 3 * n, cudaMemcpyDeviceToHost)) == cudaSuccess)
    e = cudaMemcpy(eps.data(), sim->scene.eps, 8 * n, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_error(e, "delta_sim_write_vtu: copy");
  return delta_write_vtu_host(path, step, n, pos.data(), vel.data(), eps.data());
}

}  // extern "C"
