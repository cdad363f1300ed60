// pose.cuh -- a body's current vertices formed from its reference vertices and its pose.
//
// updateVertices (dynamics.cpp:215-242) sets every vertex of a moving body to
// x = pos + R (r - ref_pos), R column-major.  posed_point is that arithmetic in xf64 (each
// operation rounded once, in the reference's order).  The vertex update kernel writes its
// result; the certified driver's kernels can instead form it where they read a vertex, so
// within a call of several time steps no vertex has to be written.
#pragma once
#include <cmath>

#include "real.cuh"

namespace delta {

// expmap, dynamics.cpp:26-102 (Taylor branch below 10 degrees; the off-diagonal term
// v02 = Omega2*Omega3 of dynamics.cpp:78 is kept as written).
__device__ __forceinline__ void expmap(xf64 O1, xf64 O2, xf64 O3, xf64 L[9]) {
  using X = xf64;
  const X v0 = O1 * O1, v1 = O2 * O2, v2 = O3 * O3;
  X angsq = v0 + v1 + v2, sx, cx;
  if (angsq < X(3.0461741978671E-02)) {
    sx = X(1.0) + (X(-1.666666666666667E-1) + (X(8.333333333333333E-3) + (X(-1.984126984126984E-4) +
         (X(2.755731922398589E-6) + (X(-2.505210838544172E-8) + X(1.605904383682161E-10) * angsq) * angsq) *
         angsq) * angsq) * angsq) * angsq;
    cx = X(0.5) + (X(-4.166666666666667E-2) + (X(1.388888888888889E-3) + (X(-2.480158730158730E-5) +
         (X(2.755731922398589E-7) + (X(-2.087675698786810E-9) + X(1.147074559772972E-11) * angsq) * angsq) *
         angsq) * angsq) * angsq) * angsq;
  } else {
    const X t = angsq;
    angsq = sqrt_(angsq);
    const X s = X(sin(angsq.v)), c = X(cos(angsq.v));
    sx = s / angsq;
    cx = (X(1.0) - c) / t;
  }
  const X v01 = O1 * O2, v02 = O2 * O3, v12 = O2 * O3;
  const X s0 = sx * O1, s1 = sx * O2, s2 = sx * O3;
  L[0] = -cx * (v2 + v1);
  L[1] = cx * v01;
  L[2] = cx * v02;
  L[3] = L[1];
  L[4] = -cx * (v2 + v0);
  L[5] = cx * v12;
  L[6] = L[2];
  L[7] = L[5];
  L[8] = -cx * (v1 + v0);
  L[0] += X(1.0);
  L[1] += s2;
  L[2] -= s1;
  L[3] -= s2;
  L[4] += X(1.0);
  L[5] += s0;
  L[6] += s1;
  L[7] -= s0;
  L[8] += X(1.0);
}


__device__ __forceinline__ void posed_point(const xf64 R[9], const xf64 pos[3], const xf64 rp[3], double r0,
                                            double r1, double r2, double out[3]) {
  const xf64 C0 = xf64(r0) - rp[0], C1 = xf64(r1) - rp[1], C2 = xf64(r2) - rp[2];
  out[0] = (pos[0] + (R[0] * C0 + R[3] * C1 + R[6] * C2)).v;
  out[1] = (pos[1] + (R[1] * C0 + R[4] * C1 + R[7] * C2)).v;
  out[2] = (pos[2] + (R[2] * C0 + R[5] * C1 + R[8] * C2)).v;
}

// The bodies' poses, for kernels that read the current vertices of a scene whose vertex
// arrays are not up to date.  rx == null: no pose, the meshes' vertices are current.
struct Pose {
  const double *rx, *ry, *rz;         // reference vertices, 3 per triangle
  const double *rot, *pos, *ref_pos;  // planes of n bodies: R (9), centre (3), reference centre (3)
  const uint8_t *obstacle;            // obstacles never move: their mesh vertices are current
  const double *reach;                // per body: max |r - ref_pos| over its reference vertices
  const double *obox;                 // per body (lo[3], hi[3]): the box of an obstacle's vertices
  int32_t n;
};

struct BodyPose {
  xf64 R[9], pos[3], rp[3];
};

__device__ __forceinline__ BodyPose body_pose(const Pose &P, int32_t b) {
  BodyPose q;
#pragma unroll
  for (int k = 0; k < 9; ++k) q.R[k] = xf64(__ldg(P.rot + (int64_t)k * P.n + b));
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    q.pos[k] = xf64(__ldg(P.pos + (int64_t)k * P.n + b));
    q.rp[k] = xf64(__ldg(P.ref_pos + (int64_t)k * P.n + b));
  }
  return q;
}

// Triangle t of a moving body with pose q: its three current vertices T[v][coordinate].
__device__ __forceinline__ void posed_tri(const Pose &P, const BodyPose &q, int64_t t, double T[3][3]) {
#pragma unroll
  for (int v = 0; v < 3; ++v)
    posed_point(q.R, q.pos, q.rp, __ldg(P.rx + 3 * t + v), __ldg(P.ry + 3 * t + v), __ldg(P.rz + 3 * t + v), T[v]);
}

// A box (lo, hi) holding every current vertex of body b.  An obstacle has its stored box.
// A moving body's vertex is pos + R C with |C| <= reach, so along axis k it lies within
// reach |row k of R| of pos_k (Cauchy-Schwarz); the half-width is widened by a relative
// 1e-9 and by 1e-12 (|pos_k| + reach), far above the rounding of the vertex arithmetic
// and of the bound itself.  A larger box only culls less, so the bound need not be tight.
__device__ __forceinline__ void pose_box(const Pose &P, int32_t b, double lo[3], double hi[3]) {
  if (P.obstacle[b]) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      lo[k] = P.obox[6 * (int64_t)b + k];
      hi[k] = P.obox[6 * (int64_t)b + 3 + k];
    }
    return;
  }
  const double reach = P.reach[b];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double r0 = P.rot[(int64_t)k * P.n + b], r1 = P.rot[(int64_t)(3 + k) * P.n + b],
                 r2 = P.rot[(int64_t)(6 + k) * P.n + b];
    const double c = P.pos[(int64_t)k * P.n + b];
    const double h = reach * sqrt(r0 * r0 + r1 * r1 + r2 * r2) * (1.0 + 1e-9) + 1e-12 * (fabs(c) + reach);
    lo[k] = c - h;
    hi[k] = c + h;
  }
}

}  // namespace delta
