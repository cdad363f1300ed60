// zoltan.cu -- the reference's zoltan/ code path on the GPU: the narrowphase with the
// "one triangle against a list" SoA shape (zoltan/bf.h, penalty.h, hybrid.h), the
// whole-system integration (zoltan/dynamics.cpp) and the contact forces
// (zoltan/forces.cpp), all FP64 over xf64 (every operation rounded once, in the
// reference's order).  Arrays are device pointers given as the reference's pointer arrays
// (d[k] = coordinate k of every list entry; t[v][k] = coordinate k of vertex v of every
// triangle, v = 0..2 spatial and 3..5 referential).
#include <cub/cub.cuh>

#include "internal.h"
#include "pose.cuh"
#include "tri_zoltan.cuh"

namespace delta {
namespace {

using X = xf64;

struct Tri3 {
  double v[3][3];  // a, b, c
};
struct ZList {
  const double *d[3], *e[3], *f[3];
  double *p[3], *q[3];
};

__device__ __forceinline__ void load_entry(const ZList &L, uint32_t i, X D[3], X E[3], X F[3]) {
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    D[k] = X(L.d[k][i]);
    E[k] = X(L.e[k][i]);
    F[k] = X(L.f[k][i]);
  }
}

__device__ __forceinline__ void store_entry(const ZList &L, uint32_t i, const X P[3], const X Q[3]) {
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    L.p[k][i] = P[k].v;
    L.q[k][i] = Q[k].v;
  }
}

// bf(it, nt, ...): the per-pair zoltan bf of triangle abc against list entry i, i in
// [it, nt); entries where it returns early keep their p, q.
__global__ void k_zoltan_bf(uint32_t it, uint32_t nt, Tri3 abc, ZList L) {
  const uint32_t i = it + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nt) return;
  X A[3][3], B[3][3];
#pragma unroll
  for (int v = 0; v < 3; ++v)
#pragma unroll
    for (int k = 0; k < 3; ++k) A[v][k] = X(abc.v[v][k]);
  load_entry(L, i, B[0], B[1], B[2]);
  X pq[6];
  if (zoltan::bf_pair(A, B, pq)) return;
  store_entry(L, i, pq, pq + 3);
}

__global__ void k_zoltan_penalty(uint32_t it, uint32_t nt, Tri3 abc, ZList L) {
  const uint32_t i = it + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nt) return;
  X A[3], Bv[3], Cv[3], D[3], E[3], F[3], P[3], Q[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    A[k] = X(abc.v[0][k]);
    Bv[k] = X(abc.v[1][k]);
    Cv[k] = X(abc.v[2][k]);
  }
  load_entry(L, i, D, E, F);
  zoltan::penalty5(A, Bv, Cv, D, E, F, i, P, Q);
  store_entry(L, i, P, Q);
}

// hybrid(it, nt, ...): one thread per batch k in [it, nt/4) of the entries 4k..4k+3.
// The batch's penalty points, then, when the mean error of its 4 entries exceeds 1e-8,
// the points of bf with the batch's last entry for all 4 (zoltan/hybrid.cpp:106-129).
// The serial loop carries P and Q from call to call; bf with the same input gives the
// same points each time, so one evaluation serves the batch.
__global__ void k_zoltan_hybrid(uint32_t k0, uint32_t k1, Tri3 abc, ZList L) {
  const uint32_t k = k0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= k1) return;
  X A[3], Bv[3], Cv[3], D[3], E[3], F[3], P[3], Q[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    A[c] = X(abc.v[0][c]);
    Bv[c] = X(abc.v[1][c]);
    Cv[c] = X(abc.v[2][c]);
  }
  X err[4];
  for (uint32_t l = 0; l < 4; ++l) {
    const uint32_t i = 4 * k + l;
    load_entry(L, i, D, E, F);
    err[l] = zoltan::penalty7(A, Bv, Cv, D, E, F, P, Q);
    store_entry(L, i, P, Q);
  }
  X batch = X(0.0);
#pragma unroll
  for (int l = 0; l < 4; ++l) batch = batch + err[l];
  if (batch / X(4.0) > X(1E-8)) {
    zoltan::hybrid_bf(A, Bv, Cv, D, E, F, P, Q);
    for (uint32_t l = 0; l < 4; ++l) store_entry(L, 4 * k + l, P, Q);
  }
}

// ---- dynamics -------------------------------------------------------------------------
struct ZBodies {
  double *angular[6], *linear[3], *rotation[9], *position[6];
  const double *inertia[9], *inverse[9], *mass;
  double *force[3], *torque[3];
};
struct ZTris {
  double *t[6][3];
  const int32_t *pid;
};

__device__ __forceinline__ void tvmul(const X *A, const X *B, X *C) {
  C[0] = A[0] * B[0] + A[1] * B[1] + A[2] * B[2];
  C[1] = A[3] * B[0] + A[4] * B[1] + A[5] * B[2];
  C[2] = A[6] * B[0] + A[7] * B[1] + A[8] * B[2];
}
__device__ __forceinline__ void nvmul(const X *A, const X *B, X *C) {
  C[0] = A[0] * B[0] + A[3] * B[1] + A[6] * B[2];
  C[1] = A[1] * B[0] + A[4] * B[1] + A[7] * B[2];
  C[2] = A[2] * B[0] + A[5] * B[1] + A[8] * B[2];
}
__device__ __forceinline__ void nnmul(const X *A, const X *B, X *C) {
#pragma unroll
  for (int col = 0; col < 3; ++col)
#pragma unroll
    for (int row = 0; row < 3; ++row)
      C[3 * col + row] = A[row] * B[3 * col] + A[3 + row] * B[3 * col + 1] + A[6 + row] * B[3 * col + 2];
}
// NVADDMUL(C, A, B, D) of zoltan/algo.h: D = C + (A B), the product summed first
__device__ __forceinline__ void nvaddmul(const X *C, const X *A, const X *B, X *D) {
  const X d0 = C[0] + (A[0] * B[0] + A[3] * B[1] + A[6] * B[2]);
  const X d1 = C[1] + (A[1] * B[0] + A[4] * B[1] + A[7] * B[2]);
  const X d2 = C[2] + (A[2] * B[0] + A[5] * B[1] + A[8] * B[2]);
  D[0] = d0;
  D[1] = d1;
  D[2] = d2;
}

// dynamics::update's body loop, zoltan/dynamics.cpp:75-188
__global__ void k_zoltan_update_bodies(int32_t nb, ZBodies s, double step_) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  const X step = X(step_), half = X(0.5) * step;
  X O[3], v[3], L1[9], J[9], I[9], f[3], tq[3], T[3], DL[9], L2[9], A[3], B[3], o[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    O[k] = X(s.angular[k][i]);
    v[k] = X(s.linear[k][i]);
    f[k] = X(s.force[k][i]);
    tq[k] = X(s.torque[k][i]);
    s.force[k][i] = 0.0;
    s.torque[k][i] = 0.0;
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    L1[k] = X(s.rotation[k][i]);
    J[k] = X(s.inertia[k][i]);
    I[k] = X(s.inverse[k][i]);
  }
  X im = X(1.0) / X(s.mass[i]);
  tvmul(L1, tq, T);
  expmap(-half * O[0], -half * O[1], -half * O[2], DL);
  nvmul(J, O, A);
  nvmul(DL, A, B);
#pragma unroll
  for (int k = 0; k < 3; ++k) B[k] = B[k] + half * T[k];
  nvmul(I, B, A);
  nvmul(J, A, B);
  T[0] -= A[1] * B[2] - A[2] * B[1];
  T[1] -= A[2] * B[0] - A[0] * B[2];
  T[2] -= A[0] * B[1] - A[1] * B[0];
#pragma unroll
  for (int k = 0; k < 3; ++k) T[k] *= step;
  nvaddmul(O, I, T, O);
  im *= step;
#pragma unroll
  for (int k = 0; k < 3; ++k) v[k] = v[k] + im * f[k];
  expmap(step * O[0], step * O[1], step * O[2], DL);
  nnmul(L1, DL, L2);
#pragma unroll
  for (int k = 0; k < 9; ++k) s.rotation[k][i] = L2[k].v;
  nvmul(L2, O, o);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    s.position[k][i] = (X(s.position[k][i]) + step * v[k]).v;
    s.angular[k][i] = O[k].v;
    s.angular[3 + k][i] = o[k].v;
    s.linear[k][i] = v[k].v;
  }
}

// dynamics::update's triangle loop, zoltan/dynamics.cpp:190-249: spatial vertices from
// the referential ones, x + L (X_ref - X_centre) (SCC, then NVADDMUL).
__global__ void k_zoltan_update_tris(int32_t nt, ZTris tr, ZBodies s, int32_t nb) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nt) return;
  const int32_t j = tr.pid[i];
  if (j < 0 || j >= nb) return;
  X L[9], Xc[3], x[3], C[3], c[3];
#pragma unroll
  for (int k = 0; k < 9; ++k) L[k] = X(s.rotation[k][j]);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    Xc[k] = X(s.position[3 + k][j]);
    x[k] = X(s.position[k][j]);
  }
#pragma unroll
  for (int w = 0; w < 3; ++w) {
#pragma unroll
    for (int k = 0; k < 3; ++k) C[k] = X(tr.t[3 + w][k][i]) - Xc[k];
    nvaddmul(x, L, C, c);
#pragma unroll
    for (int k = 0; k < 3; ++k) tr.t[w][k][i] = c[k].v;
  }
}

// dynamics::euler, zoltan/dynamics.cpp:252-297
__global__ void k_zoltan_euler(int32_t nb, ZBodies s, double step_) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  const X step = X(step_);
  X O[3], L1[9], DL[9], L2[9], o[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) O[k] = X(s.angular[k][i]);
  expmap(step * O[0], step * O[1], step * O[2], DL);
#pragma unroll
  for (int k = 0; k < 9; ++k) L1[k] = X(s.rotation[k][i]);
  nnmul(L1, DL, L2);
#pragma unroll
  for (int k = 0; k < 9; ++k) s.rotation[k][i] = L2[k].v;
  nvmul(L2, O, o);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    s.angular[3 + k][i] = o[k].v;
    s.position[k][i] = (X(s.position[k][i]) + step * X(s.linear[k][i])).v;
  }
}

// dynamics::integrate, zoltan/dynamics.cpp:299-335
struct ZMove {
  double *t[3][3];
  double *v[3];
  double lo[3], hi[3];
};
__global__ void k_zoltan_integrate(int32_t nt, ZMove m, double step_) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nt) return;
  const X step = X(step_);
  X vel[3], p[3][3];
#pragma unroll
  for (int k = 0; k < 3; ++k) vel[k] = X(m.v[k][i]);
#pragma unroll
  for (int w = 0; w < 3; ++w)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      p[w][k] = X(m.t[w][k][i]) + step * vel[k];
      m.t[w][k][i] = p[w][k].v;
    }
#pragma unroll
  for (int w = 0; w < 3; ++w) {
#pragma unroll
    for (int k = 0; k < 3; ++k)
      if (p[w][k].v < m.lo[k]) vel[k] = -vel[k];
#pragma unroll
    for (int k = 0; k < 3; ++k)
      if (p[w][k].v > m.hi[k]) vel[k] = -vel[k];
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) m.v[k][i] = vel[k].v;
}

// ---- forces -------------------------------------------------------------------------
struct ZContacts {
  const int64_t *offset;  // [nb+1] contacts of master i: [offset[i], offset[i+1])
  const int32_t *slave;
  const double *point[3], *normal[3], *depth;
};
struct ZState {
  const double *position[3], *angular[3], *linear[3], *mass;  // angular: the spatial part (angular[3..5])
  double *force[3], *torque[3];
  double gravity[3], spring, damper;
};

// granular's force on the master of contact c (zoltan/forces.cpp:28-44 with the relative
// velocity of forces.cpp:75-107).
__device__ __forceinline__ void contact_force(const ZContacts &C, const ZState &S, int32_t i, int64_t c, X f[3]) {
  X p[3], n[3], z[3], vi[3], vj[3], vij[3], oi[3], oj[3], xi[3];
  const int32_t j = C.slave[c];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    p[k] = X(C.point[k][c]);
    n[k] = X(C.normal[k][c]);
    xi[k] = X(S.position[k][i]);
    oi[k] = X(S.angular[k][i]);
    oj[k] = X(S.angular[k][j]);
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) z[k] = p[k] - xi[k];
  vi[0] = oi[1] * z[2] - oi[2] * z[1] + X(S.linear[0][i]);
  vi[1] = oi[2] * z[0] - oi[0] * z[2] + X(S.linear[1][i]);
  vi[2] = oi[0] * z[1] - oi[1] * z[0] + X(S.linear[2][i]);
#pragma unroll
  for (int k = 0; k < 3; ++k) z[k] = p[k] - X(S.position[k][j]);
  vj[0] = oj[1] * z[2] - oj[2] * z[1] + X(S.linear[0][j]);
  vj[1] = oj[2] * z[0] - oj[0] * z[2] + X(S.linear[1][j]);
  vj[2] = oj[0] * z[1] - oj[1] * z[0] + X(S.linear[2][j]);
#pragma unroll
  for (int k = 0; k < 3; ++k) vij[k] = vj[k] - vi[k];
  const X ma = X(1.0) / ((X(1.0) / X(S.mass[i])) + (X(1.0) / X(S.mass[j])));
  const X kn = X(S.spring);
  const X en = X(S.damper) * sqrt_(kn * ma);
  const X vn = dot3(vij, n);
  const X fn = (kn * X(C.depth[c])) + (en * vn);
#pragma unroll
  for (int k = 0; k < 3; ++k) f[k] = fn * n[k];
}

// Adds f (and the torque of f about body b's position, arm p - x_b) to F, T.
__device__ __forceinline__ void add_term(const ZContacts &C, const ZState &S, int32_t b, int64_t c, const X f[3],
                                         X F[3], X T[3]) {
  X a[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    F[k] += f[k];
    a[k] = X(C.point[k][c]) - X(S.position[k][b]);
  }
  T[0] += a[1] * f[2] - a[2] * f[1];
  T[1] += a[2] * f[0] - a[0] * f[2];
  T[2] += a[0] * f[1] - a[1] * f[0];
}

// One thread per body b: the additions of forces::force in the order the serial loop
// makes them on b -- the contacts in which b is the slave and the master comes first
// (-f), b's own contacts (+f; a contact with itself as slave also -f right after), the
// gravity, then the contacts in which b is the slave and the master comes later.
// by_slave[] lists the contact indices ordered by (slave, index); range [s0, s1) is b's.
// A contact whose slave is not a body index (0 <= slave < nb) adds nothing.
__device__ __forceinline__ int32_t master_of(const ZContacts &C, int32_t nb, int64_t c) {
  int32_t l = 0, h = nb;  // the body whose range [offset[l], offset[l+1]) holds c
  while (l < h) {
    const int32_t mid = (l + h) >> 1;
    if (C.offset[mid + 1] <= c) l = mid + 1;
    else h = mid;
  }
  return l < nb ? l : nb - 1;
}

__global__ void k_zoltan_force_sums(int32_t nb, ZContacts C, ZState S, const uint32_t *by_slave,
                                    const uint32_t *slave_sorted, int64_t nc) {
  const int32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  int64_t lo = 0, hi = nc;  // first entry with slave >= b
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (slave_sorted[mid] < (uint32_t)b) lo = mid + 1;
    else hi = mid;
  }
  const int64_t own0 = max((int64_t)0, C.offset[b]), own1 = min(nc, C.offset[b + 1]);
  X F[3], T[3], f[3], g[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    F[k] = X(S.force[k][b]);
    T[k] = X(S.torque[k][b]);
  }
  int64_t e = lo;
  for (; e < nc && slave_sorted[e] == (uint32_t)b; ++e) {  // masters before b
    const int64_t c = by_slave[e];
    if (c >= own0) break;
    contact_force(C, S, master_of(C, nb, c), c, f);
#pragma unroll
    for (int k = 0; k < 3; ++k) g[k] = -f[k];
    add_term(C, S, b, c, g, F, T);
  }
  for (int64_t c = own0; c < own1; ++c) {  // b's own contacts
    if (C.slave[c] < 0 || C.slave[c] >= nb) continue;
    contact_force(C, S, b, c, f);
    add_term(C, S, b, c, f, F, T);
    if (C.slave[c] == b) {
#pragma unroll
      for (int k = 0; k < 3; ++k) g[k] = -f[k];
      add_term(C, S, b, c, g, F, T);
    }
  }
  const X mb = X(S.mass[b]);
#pragma unroll
  for (int k = 0; k < 3; ++k) F[k] += mb * X(S.gravity[k]);
  for (; e < nc && slave_sorted[e] == (uint32_t)b; ++e) {  // masters after b (own-range entries skipped)
    const int64_t c = by_slave[e];
    if (c < own1) continue;
    contact_force(C, S, master_of(C, nb, c), c, f);
#pragma unroll
    for (int k = 0; k < 3; ++k) g[k] = -f[k];
    add_term(C, S, b, c, g, F, T);
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    S.force[k][b] = F[k].v;
    S.torque[k][b] = T[k].v;
  }
}

__global__ void k_iota_u32(uint32_t *v, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = (uint32_t)i;
}

inline unsigned blocks_for(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

bool all3(const void *const *p, int n) {
  for (int k = 0; k < n; ++k)
    if (!p[k]) return false;
  return true;
}

delta_status zoltan_narrow(delta_ctx *ctx, int method, int64_t it, int64_t nt, const double a[3],
                           const double b[3], const double c[3], const double *const d[3], const double *const e[3],
                           const double *const f[3], double *const p[3], double *const q[3]) {
  if (!ctx) return set_error(DELTA_ERR_INVALID, "null context");
  if (it < 0 || nt < 0) return set_error(DELTA_ERR_INVALID, "zoltan: it and nt must be >= 0");
  int64_t lo = it, hi = nt;  // threads over [lo, hi): list entries, or batches for hybrid
  if (method == 2) hi = nt / 4;
  if (hi <= lo) return DELTA_OK;
  if (!a || !b || !c || !d || !e || !f || !p || !q) return set_error(DELTA_ERR_INVALID, "zoltan: null argument");
  if (!all3((const void *const *)d, 3) || !all3((const void *const *)e, 3) || !all3((const void *const *)f, 3) ||
      !all3((const void *const *)p, 3) || !all3((const void *const *)q, 3))
    return set_error(DELTA_ERR_INVALID, "zoltan: null list pointer");
  Tri3 abc;
  for (int k = 0; k < 3; ++k) {
    abc.v[0][k] = a[k];
    abc.v[1][k] = b[k];
    abc.v[2][k] = c[k];
  }
  ZList L;
  for (int k = 0; k < 3; ++k) {
    L.d[k] = d[k];
    L.e[k] = e[k];
    L.f[k] = f[k];
    L.p[k] = p[k];
    L.q[k] = q[k];
  }
  const int threads = 128;
  const unsigned grid = blocks_for(hi - lo, threads);
  if (method == 0) k_zoltan_bf<<<grid, threads, 0, ctx->stream>>>((uint32_t)lo, (uint32_t)hi, abc, L);
  else if (method == 1) k_zoltan_penalty<<<grid, threads, 0, ctx->stream>>>((uint32_t)lo, (uint32_t)hi, abc, L);
  else k_zoltan_hybrid<<<grid, threads, 0, ctx->stream>>>((uint32_t)lo, (uint32_t)hi, abc, L);
  ctx->launches += 1;
  return cuda_error(cudaGetLastError(), "zoltan narrowphase launch");
}

}  // namespace
}  // namespace delta

using namespace delta;

extern "C" {

delta_status delta_zoltan_bf(delta_ctx *ctx, uint32_t it, uint32_t nt, const double a[3], const double b[3],
                             const double c[3], const double *const d[3], const double *const e[3],
                             const double *const f[3], double *const p[3], double *const q[3]) {
  return zoltan_narrow(ctx, 0, it, nt, a, b, c, d, e, f, p, q);
}

delta_status delta_zoltan_penalty(delta_ctx *ctx, uint32_t it, uint32_t nt, const double a[3], const double b[3],
                                  const double c[3], const double *const d[3], const double *const e[3],
                                  const double *const f[3], double *const p[3], double *const q[3]) {
  return zoltan_narrow(ctx, 1, it, nt, a, b, c, d, e, f, p, q);
}

delta_status delta_zoltan_hybrid(delta_ctx *ctx, int32_t it, int32_t nt, const double a[3], const double b[3],
                                 const double c[3], const double *const d[3], const double *const e[3],
                                 const double *const f[3], double *const p[3], double *const q[3]) {
  return zoltan_narrow(ctx, 2, it, nt, a, b, c, d, e, f, p, q);
}

delta_status delta_zoltan_update(delta_ctx *ctx, int32_t nt, int32_t nb, double *const t[6][3], const int32_t *pid,
                                 double *const angular[6], double *const linear[3], double *const rotation[9],
                                 double *const position[6], const double *const inertia[9],
                                 const double *const inverse[9], const double *mass, double *const force[3],
                                 double *const torque[3], double step) {
  if (!ctx) return set_error(DELTA_ERR_INVALID, "null context");
  if (nt < 0 || nb < 0) return set_error(DELTA_ERR_INVALID, "delta_zoltan_update: negative size");
  if (nb == 0 && nt == 0) return DELTA_OK;
  if (!angular || !linear || !rotation || !position || !inertia || !inverse || !mass || !force || !torque ||
      (nt > 0 && (!t || !pid)))
    return set_error(DELTA_ERR_INVALID, "delta_zoltan_update: null argument");
  ZBodies s;
  for (int k = 0; k < 6; ++k) s.angular[k] = angular[k], s.position[k] = position[k];
  for (int k = 0; k < 3; ++k) s.linear[k] = linear[k], s.force[k] = force[k], s.torque[k] = torque[k];
  for (int k = 0; k < 9; ++k) s.rotation[k] = rotation[k], s.inertia[k] = inertia[k], s.inverse[k] = inverse[k];
  s.mass = mass;
  if (nb > 0) {
    k_zoltan_update_bodies<<<blocks_for(nb, 128), 128, 0, ctx->stream>>>(nb, s, step);
    ctx->launches += 1;
  }
  if (nt > 0) {
    ZTris tr;
    for (int v = 0; v < 6; ++v)
      for (int k = 0; k < 3; ++k) tr.t[v][k] = t[v][k];
    tr.pid = pid;
    k_zoltan_update_tris<<<blocks_for(nt, 128), 128, 0, ctx->stream>>>(nt, tr, s, nb);
    ctx->launches += 1;
  }
  return cuda_error(cudaGetLastError(), "delta_zoltan_update launch");
}

delta_status delta_zoltan_euler(delta_ctx *ctx, int32_t nb, double *const angular[6], const double *const linear[3],
                                double *const rotation[9], double *const position[6], double step) {
  if (!ctx) return set_error(DELTA_ERR_INVALID, "null context");
  if (nb < 0) return set_error(DELTA_ERR_INVALID, "delta_zoltan_euler: negative size");
  if (nb == 0) return DELTA_OK;
  if (!angular || !linear || !rotation || !position)
    return set_error(DELTA_ERR_INVALID, "delta_zoltan_euler: null argument");
  ZBodies s = {};
  for (int k = 0; k < 6; ++k) s.angular[k] = angular[k], s.position[k] = position[k];
  for (int k = 0; k < 3; ++k) s.linear[k] = const_cast<double *>(linear[k]);
  for (int k = 0; k < 9; ++k) s.rotation[k] = rotation[k];
  k_zoltan_euler<<<blocks_for(nb, 128), 128, 0, ctx->stream>>>(nb, s, step);
  ctx->launches += 1;
  return cuda_error(cudaGetLastError(), "delta_zoltan_euler launch");
}

delta_status delta_zoltan_integrate(delta_ctx *ctx, double step, const double lo[3], const double hi[3], int32_t nt,
                                    double *const t[3][3], double *const v[3]) {
  if (!ctx) return set_error(DELTA_ERR_INVALID, "null context");
  if (nt < 0) return set_error(DELTA_ERR_INVALID, "delta_zoltan_integrate: negative size");
  if (nt == 0) return DELTA_OK;
  if (!lo || !hi || !t || !v) return set_error(DELTA_ERR_INVALID, "delta_zoltan_integrate: null argument");
  ZMove m;
  for (int w = 0; w < 3; ++w)
    for (int k = 0; k < 3; ++k) m.t[w][k] = t[w][k];
  for (int k = 0; k < 3; ++k) m.v[k] = v[k], m.lo[k] = lo[k], m.hi[k] = hi[k];
  k_zoltan_integrate<<<blocks_for(nt, 128), 128, 0, ctx->stream>>>(nt, m, step);
  ctx->launches += 1;
  return cuda_error(cudaGetLastError(), "delta_zoltan_integrate launch");
}

delta_status delta_zoltan_force(delta_ctx *ctx, int32_t nb, const int64_t *offset, const int32_t *slave,
                                int64_t n_contacts, const double *const point[3], const double *const normal[3],
                                const double *depth, const double *const position[6],
                                const double *const angular[6], const double *const linear[3], const double *mass,
                                double *const force[3], double *const torque[3], const double gravity[3],
                                double spring, double damper) {
  if (!ctx) return set_error(DELTA_ERR_INVALID, "null context");
  if (nb < 0 || n_contacts < 0 || n_contacts > 0xffffffffLL)
    return set_error(DELTA_ERR_INVALID, "delta_zoltan_force: bad size");
  if (nb == 0) return DELTA_OK;
  if (!offset || !position || !angular || !linear || !mass || !force || !torque || !gravity ||
      (n_contacts > 0 && (!slave || !point || !normal || !depth)))
    return set_error(DELTA_ERR_INVALID, "delta_zoltan_force: null argument");
  ZContacts C = {};
  C.offset = offset;
  C.slave = slave;
  C.depth = depth;
  ZState S = {};
  for (int k = 0; k < 3; ++k) {
    if (n_contacts > 0) {
      C.point[k] = point[k];
      C.normal[k] = normal[k];
    }
    S.position[k] = position[k];
    S.angular[k] = angular[3 + k];
    S.linear[k] = linear[k];
    S.force[k] = force[k];
    S.torque[k] = torque[k];
    S.gravity[k] = gravity[k];
  }
  S.mass = mass;
  S.spring = spring;
  S.damper = damper;
  cudaStream_t s = ctx->stream;
  const int64_t nc = n_contacts;
  // contact indices ordered by (slave, index): a stable radix sort of the slave ids as
  // unsigned keys over all 32 bits, so that ids outside [0, nb) sort past every body
  const uint32_t *ukeys = reinterpret_cast<const uint32_t *>(slave);
  size_t temp_bytes = 0;
  cudaError_t e = cudaSuccess;
  if (nc > 0)
    e = cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                        (const uint32_t *)nullptr, (uint32_t *)nullptr, (int)nc, 0, 32, s);
  if (e != cudaSuccess) return cuda_error(e, "delta_zoltan_force sort size");
  const size_t bytes = (size_t)(nc > 0 ? nc : 1) * (2 * sizeof(uint32_t) + sizeof(int32_t)) + temp_bytes + 256;
  void *scratch = nullptr;
  delta_status st = ctx_scratch(ctx, 27, bytes, &scratch);
  if (st != DELTA_OK) return st;
  uint32_t *idx_in = (uint32_t *)scratch, *idx_out = idx_in + (nc > 0 ? nc : 1);
  uint32_t *keys_out = idx_out + (nc > 0 ? nc : 1);
  void *temp = (void *)(((uintptr_t)(keys_out + (nc > 0 ? nc : 1)) + 255) & ~(uintptr_t)255);
  if (nc > 0) {
    k_iota_u32<<<blocks_for(nc, 256), 256, 0, s>>>(idx_in, nc);
    e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, ukeys, keys_out, idx_in, idx_out, (int)nc, 0, 32, s);
    if (e != cudaSuccess) return cuda_error(e, "delta_zoltan_force sort");
    ctx->launches += 5;  // the index fill and cub's radix passes
  }
  k_zoltan_force_sums<<<blocks_for(nb, 128), 128, 0, s>>>(nb, C, S, idx_out, keys_out, nc);
  ctx->launches += 1;
  return cuda_error(cudaGetLastError(), "delta_zoltan_force launch");
}

}  // extern "C"
