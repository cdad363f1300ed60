// tri_learned.cuh -- the FP32 search of the learned hybrid solver and its FP64 finish for
// one triangle pair: branch-free FP32 closest-point projections, the bfSolver feature they
// name evaluated in FP64 with the reference arithmetic (bf.cpp:586-697, 920-1090), and the
// FP64 separating-plane certificate.  Used by the pair-list kernel (mlp.cu,
// k_learned_refine) and by the learned particle driver (detect.cu).
#pragma once
#include "real.cuh"
#include "tri_cert.cuh"
#include "tri_ref.cuh"

namespace delta {

// Closest point of the triangle of frame F (first vertex V0; edges e0, e1) to X in FP32,
// branch-free: the interior solution of the 2x2 normal equations when it lies inside,
// otherwise the nearest of the three edges' clamped projections (all computed, one
// selected), so the lanes of a warp never diverge.  Barycentric (s, t).  The clamps are
// saturations, which send a degenerate edge's 0 * inf = NaN to 0 (a = 0 forces d = 0, and
// so on), so no guard is needed; the edge points are ranked by the squared distance less
// |V0 - X|^2.
__device__ __forceinline__ void closest_on_frame(const float *V0, const TriFrame &F, const float *X, float &s,
                                                 float &t) {
  float D[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) D[k] = V0[k] - X[k];
  const float a = F.a, b = F.b, c = F.c, d = dot3(F.e0, D), e = dot3(F.e1, D);
  const float si = fmaf(b, e, -c * d) * F.idet, ti = fmaf(b, d, -a * e) * F.idet;
  auto q = [&](float u, float v) { return fmaf(u, fmaf(a, u, fmaf(2.f * b, v, 2.f * d)), v * fmaf(c, v, 2.f * e)); };
  const float s0 = __saturatef(-d * F.ra);               // edge t = 0
  const float t1 = __saturatef(-e * F.rc);               // edge s = 0
  const float l2 = __saturatef((c + e - b - d) * F.rden);  // edge s + t = 1
  float best = s0 * fmaf(a, s0, 2.f * d);
  s = s0;
  t = 0.f;
  const float q1 = t1 * fmaf(c, t1, 2.f * e), q2 = q(l2, 1.f - l2);
  if (q1 < best) { best = q1; s = 0.f; t = t1; }
  if (q2 < best) { s = l2; t = 1.f - l2; }
  if (si >= 0.f && ti >= 0.f && si + ti <= 1.f) { s = si; t = ti; }
}

// FP32 squared distance of vertex-face pair (X, the triangle of frame F with first vertex
// V0); the callers only rank distances, and the square ranks them alike.
__device__ __forceinline__ float pt_dist2_frame(const float *V0, const TriFrame &F, const float *X) {
  float s, t;
  closest_on_frame(V0, F, X, s, t);
  float r2 = 0.f;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float r = fmaf(s, F.e0[k], fmaf(t, F.e1[k], V0[k] - X[k]));
    r2 = fmaf(r, r, r2);
  }
  return r2;
}

// FP32 squared distance of edge pair (TA->HA, TB->HB): clamped closest parameters,
// branch-free.
__device__ __forceinline__ float seg_seg_dist2_32(const float *HA, const float *TA, const float *HB,
                                                  const float *TB) {
  float u[3], v[3], w[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    u[k] = HA[k] - TA[k];
    v[k] = HB[k] - TB[k];
    w[k] = TA[k] - TB[k];
  }
  const float a = dot3(u, u), e = dot3(v, v), b = dot3(u, v), c = dot3(u, w), f = dot3(v, w);
  const float den = fmaf(a, e, -b * b);
  float s = den > 1e-12f * (a * e) ? __saturatef(__fdividef(fmaf(b, f, -c * e), den)) : 0.f;
  const float traw = e > 0.f ? __fdividef(fmaf(b, s, f), e) : 0.f;
  const float t = __saturatef(traw);
  const float s2 = __saturatef(__fdividef(fmaf(b, t, -c), a));  // a = 0: 0/0 -> 0
  s = traw != t ? s2 : s;
  float r2 = 0.f;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float r = fmaf(s, u[k], fmaf(-t, v[k], w[k]));
    r2 = fmaf(r, r, r2);
  }
  return r2;
}

// The two vertices of T other than vertex k (the edge opposite it, joining k+1 and k+2),
// in an order of no consequence to the FP32 edge-edge distance, with one select per
// coordinate each.
__device__ __forceinline__ void other_two(const float T[3][3], int k, float P[3], float Q[3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    P[c] = k == 0 ? T[1][c] : T[0][c];
    Q[c] = k == 2 ? T[1][c] : T[2][c];
  }
}

// First index of the largest / smallest of three values.
__device__ __forceinline__ int argmax3(float x0, float x1, float x2) {
  const int i = x1 > x0 ? 1 : 0;
  return x2 > (i ? x1 : x0) ? 2 : i;
}
__device__ __forceinline__ int argmin3(float x0, float x1, float x2) {
  const int i = x1 < x0 ? 1 : 0;
  return x2 < (i ? x1 : x0) ? 2 : i;
}

// One pair, one thread (no regrouping): the centroids as the start, `sweeps` FP32
// alternating projections, the vertex-face and edge-edge features they name (the CAND = 3
// choice of k_learned_refine), the picked feature in FP64 with bfSolver's arithmetic, and
// the certificate.  Returns true when the distance of pq is certified within rel_tol of the
// true distance.  A and B hold the FP64 vertices (vertex, coordinate).
__device__ __forceinline__ bool learned_pair_solve(const double A[3][3], const double B[3][3], int sweeps,
                                                   double rel_tol, double pq_out[6]) {
  float Af[3][3], Bf[3][3];
#pragma unroll
  for (int v = 0; v < 3; ++v)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      Af[v][k] = v == 0 ? 0.f : (float)(A[v][k] - A[0][k]);  // A0 is the origin
      Bf[v][k] = (float)(B[v][k] - A[0][k]);
    }
  float s = 1.f / 3.f, t = 1.f / 3.f, u = 1.f / 3.f, w = 1.f / 3.f;
  const TriFrame FA = tri_frame(Af), FB = tri_frame(Bf);
  for (int it = 0; it < sweeps; ++it) {
    float P[3], Q[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) P[k] = Af[0][k] + s * FA.e0[k] + t * FA.e1[k];
    closest_on_frame(Bf[0], FB, P, u, w);
#pragma unroll
    for (int k = 0; k < 3; ++k) Q[k] = Bf[0][k] + u * FB.e0[k] + w * FB.e1[k];
    closest_on_frame(Af[0], FA, Q, s, t);
  }
  const int iA = argmax3(1.f - s - t, s, t), jB = argmax3(1.f - u - w, u, w);
  const int kA = argmin3(1.f - s - t, s, t), kB = argmin3(1.f - u - w, u, w);
  const int ea = (kA + 1) % 3, eb = (kB + 1) % 3;
  float X1[3], X2[3], HA[3], TA[3], HB[3], TB[3];
  pick_vertex(Bf, jB, X1);
  pick_vertex(Af, iA, X2);
  const float d1 = pt_dist2_frame(Af[0], FA, X1);
  const float d2 = pt_dist2_frame(Bf[0], FB, X2);
  const bool faceB = d2 < d1;
  const int vtx = faceB ? iA : jB;
  const float dpt = faceB ? d2 : d1;
  other_two(Af, kA, HA, TA);  // edge ea of A
  other_two(Bf, kB, HB, TB);  // edge eb of B
  const float de = seg_seg_dist2_32(HA, TA, HB, TB);
  xf64 A64[3][3], B64[3][3], pq[6];
#pragma unroll
  for (int v = 0; v < 3; ++v)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      A64[v][k] = xf64(A[v][k]);
      B64[v][k] = xf64(B[v][k]);
    }
  if (dpt > de) {  // the edge pair: seg_seg_ref, then bf.cpp:715-879's points
    xf64 H1[3], T1[3], H2[3], T2[3], sc, tc;
    pick_vertex(A64, ea, H1);
    pick_vertex(A64, (ea + 1) % 3, T1);
    pick_vertex(B64, eb, H2);
    pick_vertex(B64, (eb + 1) % 3, T2);
    seg_seg_ref(H1, T1, H2, T2, sc, tc);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      pq[k] = T1[k] + ((H1[k] - T1[k]) * sc);
      pq[3 + k] = T2[k] + ((H2[k] - T2[k]) * tc);
    }
  } else {  // the vertex-face pair: pt_tri_ref, then bf.cpp:1104-1177's points
    xf64 X[3], sf, tf;
    pick_vertex(faceB ? A64 : B64, vtx, X);
    const xf64(*F)[3] = faceB ? B64 : A64;
    pt_tri_ref(F[0], F[1], F[2], X, sf, tf);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const xf64 fp = F[0][k] + ((F[2][k] - F[0][k]) * tf) + ((F[1][k] - F[0][k]) * sf);
      pq[k] = faceB ? X[k] : fp;
      pq[3 + k] = faceB ? fp : X[k];
    }
  }
  const double d = pq_distance(pq).v;
#pragma unroll
  for (int k = 0; k < 6; ++k) pq_out[k] = pq[k].v;
  if (!(d > 0)) return false;
  const double r[3] = {pq[0].v - pq[3].v, pq[1].v - pq[4].v, pq[2].v - pq[5].v};
  double amin = 1e300, bmax = -1e300, scale = 0.0;
#pragma unroll
  for (int v = 0; v < 3; ++v) {
    amin = fmin(amin, A[v][0] * r[0] + A[v][1] * r[1] + A[v][2] * r[2]);
    bmax = fmax(bmax, B[v][0] * r[0] + B[v][1] * r[1] + B[v][2] * r[2]);
#pragma unroll
    for (int k = 0; k < 3; ++k) scale = fmax(scale, fmax(fabs(A[v][k]), fabs(B[v][k])));
  }
  const double d2r = d * d;
  return d2r - (amin - bmax) + 1e-14 * scale * d <= rel_tol * d2r;
}

}  // namespace delta
