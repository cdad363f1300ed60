// sphere.cu -- the reference's sphere contact model on the GPU (sphere.cpp, point.cpp).
//
// sphere() (sphere.cpp:29-77): two spheres given by centre and diameter touch through
// their surface points along the centre line; sphereWithBarrierAB/BA (sphere.cpp:79-201):
// a sphere against every triangle of a mesh through point.cpp's closest point pt();
// isSphereOverlayInContact (sphere.cpp:203-218): the halo-sphere overlap test.  All FP64
// arithmetic is xf64 (every operation rounded once, no contraction) in the reference's
// operation order, so contacts equal the reference's bit for bit.  Contacts are written in
// the reference's order (pair order; triangle order within a pair) by flag, scan, write.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>

#include "internal.h"
#include "real.cuh"
#include "tri_ref.cuh"

namespace delta {
namespace {

// point.cpp:11-210: closest point tq of triangle (T1,T2,T3) to c; returns the distance.
// Eberly's regions are tri_ref.cuh's, with point.cpp's `< 0` clamp.
__device__ xf64 pt_point(const xf64 T1[3], const xf64 T2[3], const xf64 T3[3], const xf64 c[3], xf64 tq[3]) {
  xf64 s, t;
  const xf64 dist = pt_tri_ref<xf64, false>(T1, T2, T3, c, s, t);
#pragma unroll
  for (int k = 0; k < 3; ++k) tq[k] = T1[k] + ((T3[k] - T1[k]) * t) + ((T2[k] - T1[k]) * s);
  return dist;
}

struct Rec {
  xf64 P[3], Q[3], epsA, epsB;
  int32_t idA, idB;
  uint8_t fric;
};

// |Q - P| as contactpoint::getDistance
__device__ __forceinline__ xf64 rec_distance(const Rec &r) {
  return sqrt_(((r.Q[0] - r.P[0]) * (r.Q[0] - r.P[0])) + ((r.Q[1] - r.P[1]) * (r.Q[1] - r.P[1])) +
               ((r.Q[2] - r.P[2]) * (r.Q[2] - r.P[2])));
}

// contactpoint(PA, epsA, idA, QB, epsB, idB, friction), contactpoint.cpp:116-155
__device__ void write_rec(const delta_contacts &o, int64_t pos, const Rec &r, int32_t tri_b) {
  const int64_t cap = o.capacity;
  const xf64 two(2.0), eps_total = r.epsA + r.epsB, dist = rec_distance(r);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    o.x[k * cap + pos] = ((r.P[k] + r.Q[k]) / two).v;
    o.normal[k * cap + pos] = ((r.P[k] - r.Q[k]) / dist).v;
    o.P[k * cap + pos] = r.P[k].v;
    o.Q[k * cap + pos] = r.Q[k].v;
  }
  o.depth[pos] = (eps_total - dist).v;
  o.eps_total[pos] = eps_total.v;
  o.master[pos] = r.idA;
  o.slave[pos] = r.idB;
  o.tri_a[pos] = -1;
  o.tri_b[pos] = tri_b;
  o.penetration[pos] = 1;
  o.friction[pos] = r.fric;
}

__device__ __forceinline__ void load_centre(const delta_spheres &s, int64_t i, xf64 c[3]) {
#pragma unroll
  for (int k = 0; k < 3; ++k) c[k] = xf64(s.centre[k * s.n + i]);
}

// sphere.cpp:46-76
__device__ bool sphere_rec(const delta_spheres &s, int32_t a, int32_t b, Rec &r) {
  xf64 cA[3], cB[3];
  load_centre(s, a, cA);
  load_centre(s, b, cB);
  const xf64 two(2.0), dA = xf64(s.diameter[a]), dB = xf64(s.diameter[b]);
  const xf64 distance = sqrt_(((cB[0] - cA[0]) * (cB[0] - cA[0])) + ((cB[1] - cA[1]) * (cB[1] - cA[1])) +
                              ((cB[2] - cA[2]) * (cB[2] - cA[2])));
  const xf64 inv = xf64(1.0) / distance;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const xf64 nk = inv * (cB[k] - cA[k]);
    r.P[k] = cA[k] + ((dA / two) * nk);
    r.Q[k] = cB[k] - ((dB / two) * nk);
  }
  r.epsA = xf64(s.eps[a]);
  r.epsB = xf64(s.eps[b]);
  r.idA = s.id[a];
  r.idB = s.id[b];
  r.fric = (s.friction[a] && s.friction[b]) ? 1 : 0;
  return rec_distance(r) <= (r.epsA + r.epsB);
}

// sphere.cpp:112-135 (sphere is A) and 175-197 (sphere is B: the mesh point comes first,
// with the sphere's epsilon and id)
__device__ bool sphere_tri_rec(const delta_spheres &s, int32_t si, const delta_meshes &m, int32_t body, int64_t t,
                               int sphere_is_b, Rec &r) {
  xf64 c[3], T[3][3], Q[3], S[3];
  load_centre(s, si, c);
  const int64_t g = m.tri_offset[body] + t;
#pragma unroll
  for (int v = 0; v < 3; ++v) {
    T[v][0] = xf64(m.x[3 * g + v]);
    T[v][1] = xf64(m.y[3 * g + v]);
    T[v][2] = xf64(m.z[3 * g + v]);
  }
  const xf64 two(2.0), d = xf64(s.diameter[si]);
  const xf64 distance = pt_point(T[0], T[1], T[2], c, Q) - (d / two);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const xf64 nk = (Q[k] - c[k]) / (distance + (d / two));
    S[k] = c[k] + ((d / two) * nk);
  }
  const xf64 epsS = xf64(s.eps[si]), epsM = xf64(m.eps[body]);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    r.P[k] = sphere_is_b ? Q[k] : S[k];
    r.Q[k] = sphere_is_b ? S[k] : Q[k];
  }
  r.epsA = epsS;
  r.epsB = epsM;
  r.idA = s.id[si];
  r.idB = m.id[body];
  r.fric = (s.friction[si] && m.friction[body]) ? 1 : 0;
  return rec_distance(r) <= (epsS + epsM);
}

__global__ void k_sphere_flags(const delta_spheres s, const int32_t *__restrict__ pa, const int32_t *__restrict__ pb,
                               int64_t n, uint32_t *__restrict__ flag) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Rec r;
  flag[i] = sphere_rec(s, pa[i], pb[i], r) ? 1u : 0u;
}

__global__ void k_sphere_write(const delta_spheres s, const int32_t *__restrict__ pa, const int32_t *__restrict__ pb,
                               int64_t n, const uint32_t *__restrict__ flag, const uint32_t *__restrict__ pos,
                               const delta_contacts o) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !flag[i] || pos[i] >= (uint64_t)o.capacity) return;
  Rec r;
  sphere_rec(s, pa[i], pb[i], r);
  write_rec(o, pos[i], r, -1);
}

__global__ void k_mesh_counts(const delta_meshes m, const int32_t *__restrict__ body, int64_t n,
                              int64_t *__restrict__ cnt) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) cnt[i] = m.tri_offset[body[i] + 1] - m.tri_offset[body[i]];
}

// one block per pair (grid-stride), threads over the body's triangles
template <bool WRITE>
__global__ void k_sphere_mesh(const delta_spheres s, const delta_meshes m, const int32_t *__restrict__ sph,
                              const int32_t *__restrict__ body, int64_t n, int sphere_is_b,
                              const int64_t *__restrict__ off, uint32_t *__restrict__ flag,
                              const uint32_t *__restrict__ pos, const delta_contacts o) {
  for (int64_t p = blockIdx.x; p < n; p += gridDim.x) {
    const int64_t nt = m.tri_offset[body[p] + 1] - m.tri_offset[body[p]];
    for (int64_t t = threadIdx.x; t < nt; t += blockDim.x) {
      const int64_t f = off[p] + t;
      if (WRITE && (!flag[f] || pos[f] >= (uint64_t)o.capacity)) continue;
      Rec r;
      const bool take = sphere_tri_rec(s, sph[p], m, body[p], t, sphere_is_b, r);
      if (WRITE) write_rec(o, pos[f], r, (int32_t)t);
      else flag[f] = take ? 1u : 0u;
    }
  }
}

__global__ void k_overlap(const double *__restrict__ c, int64_t ld, const double *__restrict__ radius,
                          const int32_t *__restrict__ pa, const int32_t *__restrict__ pb, int64_t n,
                          uint8_t *__restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t a = pa[i], b = pb[i];
  // sphere.cpp:214: pow(x, 2) is the correctly rounded square
  xf64 s2(0.0);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const xf64 d = xf64(c[k * ld + b]) - xf64(c[k * ld + a]);
    s2 = s2 + d * d;
  }
  out[i] = sqrt_(s2) <= (xf64(radius[a]) + xf64(radius[b])) ? 1 : 0;
}

inline unsigned nb(int64_t n, int t = 256) { return (unsigned)std::max<int64_t>(1, (n + t - 1) / t); }

bool spheres_ok(const delta_spheres *s) {
  return s && s->n > 0 && s->centre && s->diameter && s->eps && s->friction && s->id;
}
bool out_ok(const delta_contacts *o) {
  return o && o->capacity >= 0 &&
         (o->capacity == 0 || (o->x && o->normal && o->P && o->Q && o->depth && o->eps_total && o->master &&
                               o->slave && o->tri_a && o->tri_b && o->penetration && o->friction));
}

// exclusive scan of flag[0..n) into pos, total into *total (host); synchronises
delta_status scan_total(delta_ctx *ctx, const uint32_t *flag, uint32_t *pos, int64_t n, int slot, int64_t *total) {
  size_t tb = 0;
  cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, tb, flag, pos, n, ctx->stream);
  if (e != cudaSuccess) return cuda_error(e, "sphere: scan size");
  void *tmp;
  delta_status st = ctx_scratch(ctx, slot, tb + 16, &tmp);
  if (st != DELTA_OK) return st;
  if ((e = cub::DeviceScan::ExclusiveSum(tmp, tb, flag, pos, n, ctx->stream)) != cudaSuccess)
    return cuda_error(e, "sphere: scan");
  uint32_t h[2] = {0, 0};
  void *pin;
  if ((st = ctx_pinned(ctx, 8, &pin)) != DELTA_OK) return st;
  if ((e = cudaMemcpyAsync(pin, pos + n - 1, 4, cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(static_cast<char *>(pin) + 4, flag + n - 1, 4, cudaMemcpyDeviceToHost, ctx->stream)) !=
          cudaSuccess ||
      (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
    return cuda_error(e, "sphere: total");
  std::memcpy(h, pin, 8);
  *total = (int64_t)h[0] + h[1];
  return DELTA_OK;
}

}  // namespace
}  // namespace delta

using namespace delta;

extern "C" {

delta_status delta_sphere_contacts(delta_ctx *ctx, const delta_spheres *spheres, const int32_t *pair_a,
                                   const int32_t *pair_b, int64_t n_pairs, const delta_contacts *out,
                                   int64_t *n_out) {
  if (!ctx || !spheres_ok(spheres) || !out_ok(out) || !n_out || n_pairs < 0 || n_pairs >= (int64_t)UINT32_MAX ||
      (n_pairs > 0 && (!pair_a || !pair_b)))
    return set_error(DELTA_ERR_INVALID, "delta_sphere_contacts: bad argument");
  *n_out = 0;
  if (n_pairs == 0) return DELTA_OK;
  void *buf;
  delta_status st = ctx_scratch(ctx, 19, 8 * (size_t)n_pairs + 256, &buf);
  if (st != DELTA_OK) return st;
  uint32_t *flag = static_cast<uint32_t *>(buf), *pos = flag + n_pairs;
  k_sphere_flags<<<nb(n_pairs), 256, 0, ctx->stream>>>(*spheres, pair_a, pair_b, n_pairs, flag);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "delta_sphere_contacts: flags");
  int64_t total = 0;
  if ((st = scan_total(ctx, flag, pos, n_pairs, 20, &total)) != DELTA_OK) return st;
  k_sphere_write<<<nb(n_pairs), 256, 0, ctx->stream>>>(*spheres, pair_a, pair_b, n_pairs, flag, pos, *out);
  ctx->launches += 3;
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(e, "delta_sphere_contacts: write");
  *n_out = total;
  if (total > out->capacity) return set_error(DELTA_ERR_CAPACITY, "delta_sphere_contacts: contact buffer too small");
  return DELTA_OK;
}

delta_status delta_sphere_mesh_contacts(delta_ctx *ctx, const delta_spheres *spheres, const delta_meshes *meshes,
                                        const int32_t *sphere, const int32_t *body, int64_t n_pairs,
                                        int sphere_is_b, const delta_contacts *out, int64_t *n_out) {
  if (!ctx || !spheres_ok(spheres) || !meshes || !meshes->tri_offset || !meshes->x || !meshes->y || !meshes->z ||
      !meshes->eps || !meshes->friction || !meshes->id || !out_ok(out) || !n_out || n_pairs < 0 ||
      (n_pairs > 0 && (!sphere || !body)) || (sphere_is_b != 0 && sphere_is_b != 1))
    return set_error(DELTA_ERR_INVALID, "delta_sphere_mesh_contacts: bad argument");
  *n_out = 0;
  if (n_pairs == 0) return DELTA_OK;
  // per-pair triangle offsets into one flag array over all (pair, triangle)
  void *obuf;
  delta_status st = ctx_scratch(ctx, 19, 16 * (size_t)n_pairs + 256, &obuf);
  if (st != DELTA_OK) return st;
  int64_t *cnt = static_cast<int64_t *>(obuf), *off = cnt + n_pairs;
  k_mesh_counts<<<nb(n_pairs), 256, 0, ctx->stream>>>(*meshes, body, n_pairs, cnt);
  size_t tb = 0;
  cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, off, n_pairs, ctx->stream);
  void *tmp;
  if (e != cudaSuccess) return cuda_error(e, "sphere mesh: scan size");
  if ((st = ctx_scratch(ctx, 20, tb + 16, &tmp)) != DELTA_OK) return st;
  if ((e = cub::DeviceScan::ExclusiveSum(tmp, tb, cnt, off, n_pairs, ctx->stream)) != cudaSuccess)
    return cuda_error(e, "sphere mesh: offsets");
  int64_t h[2];
  void *pin;
  if ((st = ctx_pinned(ctx, 16, &pin)) != DELTA_OK) return st;
  if ((e = cudaMemcpyAsync(pin, off + n_pairs - 1, 8, cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(static_cast<char *>(pin) + 8, cnt + n_pairs - 1, 8, cudaMemcpyDeviceToHost,
                           ctx->stream)) != cudaSuccess ||
      (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
    return cuda_error(e, "sphere mesh: triangle total");
  std::memcpy(h, pin, 16);
  const int64_t T = h[0] + h[1];
  if (T == 0) return DELTA_OK;
  if (T >= (int64_t)UINT32_MAX) return set_error(DELTA_ERR_CAPACITY, "delta_sphere_mesh_contacts: too many triangles");
  void *fbuf;
  if ((st = ctx_scratch(ctx, 21, 8 * (size_t)T + 256, &fbuf)) != DELTA_OK) return st;
  uint32_t *flag = static_cast<uint32_t *>(fbuf), *pos = flag + T;
  const unsigned grid = (unsigned)std::min<int64_t>(n_pairs, (int64_t)kNumSMs * 16);
  k_sphere_mesh<false><<<grid, 128, 0, ctx->stream>>>(*spheres, *meshes, sphere, body, n_pairs, sphere_is_b, off, flag,
                                                      nullptr, *out);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(e, "sphere mesh: flags");
  int64_t total = 0;
  if ((st = scan_total(ctx, flag, pos, T, 22, &total)) != DELTA_OK) return st;
  k_sphere_mesh<true><<<grid, 128, 0, ctx->stream>>>(*spheres, *meshes, sphere, body, n_pairs, sphere_is_b, off, flag,
                                                     pos, *out);
  ctx->launches += 5;
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(e, "sphere mesh: write");
  *n_out = total;
  if (total > out->capacity)
    return set_error(DELTA_ERR_CAPACITY, "delta_sphere_mesh_contacts: contact buffer too small");
  return DELTA_OK;
}

delta_status delta_sphere_overlap(delta_ctx *ctx, const double *centre, int64_t ld, const double *radius,
                                  const int32_t *pair_a, const int32_t *pair_b, int64_t n_pairs, uint8_t *overlap) {
  if (!ctx || n_pairs < 0 || (n_pairs > 0 && (!centre || !radius || !pair_a || !pair_b || !overlap)) || ld < 0)
    return set_error(DELTA_ERR_INVALID, "delta_sphere_overlap: bad argument");
  if (n_pairs == 0) return DELTA_OK;
  k_overlap<<<nb(n_pairs), 256, 0, ctx->stream>>>(centre, ld, radius, pair_a, pair_b, n_pairs, overlap);
  ctx->launches += 1;
  return cuda_error(cudaGetLastError(), "delta_sphere_overlap");
}

}  // extern "C"
