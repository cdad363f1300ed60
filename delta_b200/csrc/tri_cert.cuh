// tri_cert.cuh -- bfSolver's result computed with an FP32 filter and FP64 finishing.
//
// bfSolver (bf.cpp:217-1178) returns the minimum over 15 features (9 edge-edge, 6
// vertex-face) under fixed tie rules.  Here, one warp handles 32 triangle pairs:
//
// 1. FP32, branch-free, in a frame centred on A's first vertex: for every feature a
//    feasible parameter point (s,t) and the point pair r = P(s,t) - Q(s,t) it defines.
//    Because the feature distance |r(s,t)| is convex in (s,t), the Frank-Wolfe bound
//        d_true >= |r| + min_{corners c of the parameter domain} grad|r| . (c - (s,t))
//    holds whatever (s,t) is, so inexact FP32 parameters only loosen the bound.  The
//    band eps = 64 u32 L (L = extent of the pair's bounding box) covers the rounding of
//    the inputs and of the FP32 arithmetic.  The reference's own FP64 vertex-face value
//    comes from a quadratic form, which may underestimate the squared distance by up to
//    32 u64 M (M bounds the form's terms); that is subtracted too.  Result: a certified
//    lower bound LB_f <= (reference FP64 value of feature f).
// 2. The feature with the smallest FP32 distance is evaluated in FP64 with the
//    reference's arithmetic; its value `best` bounds the reference minimum from above.
// 3. Every other feature with LB_f <= best is queued; the warp evaluates the queue 32
//    entries at a time (FP64, reference arithmetic, one code path per feature family).
// 4. Per pair, the candidates' FP64 values are reduced with the reference's selection
//    rule (lowest index among equal minima inside a family; vertex-face wins a tie
//    between the families), and the closest points are computed from the winner in FP64.
// Every feature attaining the reference minimum is a candidate, so the output equals
// bfSolver's bit for bit.
#pragma once
#include "tri_ref.cuh"

namespace delta {

constexpr float kU32 = 5.9604644775390625e-08f;  // 2^-24
constexpr double kU64 = 1.1102230246251565e-16;  // 2^-53

__device__ __forceinline__ float clamp01(float x) { return fminf(fmaxf(x, 0.f), 1.f); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }

// FP32 edge-edge: clamped closest parameters (segment P(s)=TA+s*u, Q(t)=TB+t*v), the
// distance of that point pair and its Frank-Wolfe lower bound.  Returns d, writes lb.
__device__ __forceinline__ float seg_seg_lb(const float *HA, const float *TA, const float *HB, const float *TB,
                                            float &lb) {
  float u[3], v[3], w[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    u[k] = HA[k] - TA[k];
    v[k] = HB[k] - TB[k];
    w[k] = TA[k] - TB[k];
  }
  const float a = dot3(u, u), e = dot3(v, v), b = dot3(u, v), c = dot3(u, w), f = dot3(v, w);
  const float den = fmaf(a, e, -b * b);
  float s = den > 1e-12f * (a * e) ? clamp01(fdiv(fmaf(b, f, -c * e), den)) : 0.f;
  const float traw = e > 0.f ? fdiv(fmaf(b, s, f), e) : 0.f;
  const float t = clamp01(traw);
  const float s2 = a > 0.f ? clamp01(fdiv(fmaf(b, t, -c), a)) : 0.f;
  s = (traw != t) ? s2 : s;
  float r[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) r[k] = fmaf(s, u[k], fmaf(-t, v[k], w[k]));
  const float r2 = dot3(r, r);
  const float inv = rsqrtf(r2);
  const float d = r2 > 0.f ? r2 * inv : 0.f;
  const float gs = dot3(r, u), gt = -dot3(r, v);
  const float gap = fminf(-gs * s, gs * (1.f - s)) + fminf(-gt * t, gt * (1.f - t));
  lb = d + gap * inv;  // NaN when r = 0: the feature stays a candidate
  return d;
}

// FP32 vertex-face: closest point of triangle (V0,V1,V2) to X chosen among the interior
// projection (when inside) and the three edges, its distance, and the Frank-Wolfe lower
// bound with the reference's quadratic-form error removed.  Returns d, writes lb.
__device__ __forceinline__ float pt_tri_lb(const float *V0, const float *V1, const float *V2, const float *X, float eps,
                                           float &lb) {
  float E0[3], E1[3], D[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    E0[k] = V1[k] - V0[k];
    E1[k] = V2[k] - V0[k];
    D[k] = V0[k] - X[k];
  }
  const float a = dot3(E0, E0), b = dot3(E0, E1), c = dot3(E1, E1), d = dot3(E0, D), e = dot3(E1, D), f = dot3(D, D);
  const float det = fmaf(a, c, -b * b);
  const float idet = fdiv(1.f, det);
  const float si = fmaf(b, e, -c * d) * idet, ti = fmaf(b, d, -a * e) * idet;
  const bool inside = si >= 0.f && ti >= 0.f && si + ti <= 1.f;
  // squared distance of parameter (s,t): |D + s E0 + t E1|^2 = f + 2(s d + t e) + s^2 a + 2 s t b + t^2 c
  auto q = [&](float s, float t) {
    return fmaf(s, fmaf(a, s, fmaf(2.f * b, t, 2.f * d)), fmaf(t, fmaf(c, t, 2.f * e), f));
  };
  const float s0 = a > 0.f ? clamp01(fdiv(-d, a)) : 0.f;  // edge t = 0
  const float t1 = c > 0.f ? clamp01(fdiv(-e, c)) : 0.f;  // edge s = 0
  const float den2 = a - 2.f * b + c;
  const float l2 = den2 > 0.f ? clamp01(fdiv(c + e - b - d, den2)) : 0.f;  // edge s + t = 1: s = l2
  float s = s0, t = 0.f, best = q(s0, 0.f);
  const float q1 = q(0.f, t1), q2 = q(l2, 1.f - l2);
  if (q1 < best) { best = q1; s = 0.f; t = t1; }
  if (q2 < best) { best = q2; s = l2; t = 1.f - l2; }
  if (inside) { s = si; t = ti; }
  float r[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) r[k] = fmaf(s, E0[k], fmaf(t, E1[k], D[k]));
  const float r2 = dot3(r, r);
  const float inv = rsqrtf(r2);
  const float dist = r2 > 0.f ? r2 * inv : 0.f;
  const float g0 = dot3(r, E0), g1 = dot3(r, E1);
  const float gap = fminf(fminf(-g0 * s - g1 * t, g0 * (1.f - s) - g1 * t), -g0 * s + g1 * (1.f - t));
  float lbt = fmaxf(dist + gap * inv - eps, 0.f);  // NaN propagates (fmaxf keeps 0): handled below
  if (!(r2 > 0.f)) lbt = 0.f;
  // reference FP64 quadratic-form error: sq_ref >= sq_true - 32 u64 M
  const float M = a + 2.f * fabsf(b) + c + 2.f * fabsf(d) + 2.f * fabsf(e) + f;
  const float lb2 = fmaf(lbt, lbt, -(float)(32.0 * kU64) * 1.0001f * M);
  lb = lb2 > 0.f ? sqrtf(lb2) : 0.f;
  return dist;
}

// A vertex (0..2) of A or B by runtime index.
template <class R>
__device__ __forceinline__ void pick_vertex(const R T[3][3], int i, R out[3]) {
#pragma unroll
  for (int k = 0; k < 3; ++k) out[k] = i == 0 ? T[0][k] : (i == 1 ? T[1][k] : T[2][k]);
}

// Reference value of feature f (runtime index) with one code path per family:
// f < 9: edge-edge (eA = f/3, eB = f%3); else vertex-face j = f-9.
__device__ __forceinline__ xf64 feature_dyn(const xf64 A[3][3], const xf64 B[3][3], int f, xf64 &p0, xf64 &p1) {
  if (f < 9) {
    const int ea = f / 3, eb = f - 3 * ea;
    xf64 HA[3], TA[3], HB[3], TB[3];
    pick_vertex(A, ea, HA);
    pick_vertex(A, ea == 2 ? 0 : ea + 1, TA);
    pick_vertex(B, eb, HB);
    pick_vertex(B, eb == 2 ? 0 : eb + 1, TB);
    return seg_seg_ref(HA, TA, HB, TB, p0, p1);
  }
  const int j = f - 9;
  const bool onA = j < 3;
  xf64 V0[3], V1[3], V2[3], X[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    V0[k] = onA ? A[0][k] : B[0][k];
    V1[k] = onA ? A[1][k] : B[1][k];
    V2[k] = onA ? A[2][k] : B[2][k];
  }
  const int xi = onA ? j : j - 3;
  if (onA) pick_vertex(B, xi, X);
  else pick_vertex(A, xi, X);
  return pt_tri_ref(V0, V1, V2, X, p0, p1);
}

// Closest points of the winning feature (runtime index), bf.cpp:715-879 and 1104-1177.
__device__ __forceinline__ void feature_points_dyn(const xf64 A[3][3], const xf64 B[3][3], int f, xf64 p0, xf64 p1,
                                                   double pq[6]) {
  if (f < 9) {
    const int ea = f / 3, eb = f - 3 * ea;
    xf64 HA[3], TA[3], HB[3], TB[3];
    pick_vertex(A, ea, HA);
    pick_vertex(A, ea == 2 ? 0 : ea + 1, TA);
    pick_vertex(B, eb, HB);
    pick_vertex(B, eb == 2 ? 0 : eb + 1, TB);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      pq[k] = (TA[k] + ((HA[k] - TA[k]) * p0)).v;
      pq[3 + k] = (TB[k] + ((HB[k] - TB[k]) * p1)).v;
    }
    return;
  }
  const int j = f - 9;
  const bool onA = j < 3;
  xf64 X[3], face[3];
  if (onA) pick_vertex(B, j, X);
  else pick_vertex(A, j - 3, X);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const xf64 v0 = onA ? A[0][k] : B[0][k], v1 = onA ? A[1][k] : B[1][k], v2 = onA ? A[2][k] : B[2][k];
    face[k] = v0 + ((v2 - v0) * p1) + ((v1 - v0) * p0);
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    pq[k] = onA ? face[k].v : X[k].v;
    pq[3 + k] = onA ? X[k].v : face[k].v;
  }
}

// Per-warp shared staging for bf_cert_warp: the 32 pairs' coordinates and the queue.
struct CertWarpSmem {
  double coords[32][18];
  uint16_t queue[32 * 15];
};

// Running minimum of one feature family, ordered by (distance, feature index).
struct FamilyBest {
  xf64 dist, p0, p1;
  int f;
  __device__ __forceinline__ void offer(xf64 d, int ff, xf64 a, xf64 b) {
    if (d < dist || (d == dist && ff < f)) { dist = d; f = ff; p0 = a; p1 = b; }
  }
};

// All 32 lanes call this together; lanes with valid == false carry dummy data and
// produce nothing.  Writes bfSolver's closest points to pq; returns the number of FP64
// feature evaluations made for this lane's pair.
__device__ __forceinline__ int bf_cert_warp(const double A64[3][3], const double B64[3][3], bool valid, double pq[6],
                                            CertWarpSmem &sm) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  // ---- 1. FP32 lower bounds -------------------------------------------------------
  float A[3][3], B[3][3];
  double L = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double lo = A64[0][k], hi = A64[0][k];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      A[v][k] = (float)(A64[v][k] - A64[0][k]);
      B[v][k] = (float)(B64[v][k] - A64[0][k]);
      lo = fmin(lo, fmin(A64[v][k], B64[v][k]));
      hi = fmax(hi, fmax(A64[v][k], B64[v][k]));
    }
    L = fmax(L, hi - lo);
  }
  const float eps = (float)L * (64.f * kU32);
  float d32[15], lb[15];
#pragma unroll
  for (int j = 0; j < 9; ++j) {
    float l;
    d32[j] = seg_seg_lb(A[j / 3], A[(j / 3 + 1) % 3], B[j % 3], B[(j % 3 + 1) % 3], l);
    lb[j] = l - eps;
  }
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    d32[9 + j] = pt_tri_lb(A[0], A[1], A[2], B[j], eps, lb[9 + j]);
    d32[12 + j] = pt_tri_lb(B[0], B[1], B[2], A[j], eps, lb[12 + j]);
  }
  int fmin_ = 0;
  float dmin = d32[0];
#pragma unroll
  for (int f = 1; f < 15; ++f)
    if (d32[f] < dmin) { dmin = d32[f]; fmin_ = f; }
  // ---- 2. FP64 value of the FP32 argmin ---------------------------------------------
  xf64 Ax[3][3], Bx[3][3];
#pragma unroll
  for (int v = 0; v < 3; ++v)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      Ax[v][k] = xf64(A64[v][k]);
      Bx[v][k] = xf64(B64[v][k]);
    }
  xf64 c0, c1;
  const xf64 best = feature_dyn(Ax, Bx, fmin_, c0, c1);
  FamilyBest seg{xf64(1E+30), xf64(0.0), xf64(0.0), 0}, pt{xf64(1E30), xf64(0.0), xf64(0.0), 0};
  // the reference's initial state is (1e30, first index, zero parameters); a feature
  // reaching 1e30 exactly never replaces it (strict <), which offer() reproduces by
  // treating the initial entry as index -1 only for strictly smaller distances.
  if (fmin_ < 9) { if (best < seg.dist) { seg.dist = best; seg.f = fmin_; seg.p0 = c0; seg.p1 = c1; } }
  else { if (best < pt.dist) { pt.dist = best; pt.f = fmin_ - 9; pt.p0 = c0; pt.p1 = c1; } }
  // ---- 3. queue the remaining candidates ----------------------------------------------
  unsigned mask = 0;
#pragma unroll
  for (int f = 0; f < 15; ++f)
    if (f != fmin_ && !((double)lb[f] > best.v)) mask |= 1u << f;
  if (!valid) mask = 0;
  const int cnt = __popc(mask);
  int incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(full, incl, o);
    if (lane >= o) incl += y;
  }
  const int total = __shfl_sync(full, incl, 31);
  int pos = incl - cnt;
  for (unsigned m = mask; m; m &= m - 1) sm.queue[pos++] = (uint16_t)((lane << 4) | (__ffs(m) - 1));
#pragma unroll
  for (int v = 0; v < 3; ++v)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      sm.coords[lane][3 * v + k] = A64[v][k];
      sm.coords[lane][9 + 3 * v + k] = B64[v][k];
    }
  __syncwarp();
  // ---- 3b. evaluate the queue 32 entries at a time, merge into the owners' minima -----
  for (int c = 0; c < total; c += 32) {
    const int j = c + lane;
    int owner = 0, f = 0;
    xf64 dist = xf64(0.0), p0 = xf64(0.0), p1 = xf64(0.0);
    if (j < total) {
      const uint16_t e = sm.queue[j];
      owner = e >> 4;
      f = e & 15;
      xf64 QA[3][3], QB[3][3];
#pragma unroll
      for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          QA[v][k] = xf64(sm.coords[owner][3 * v + k]);
          QB[v][k] = xf64(sm.coords[owner][9 + 3 * v + k]);
        }
      dist = feature_dyn(QA, QB, f, p0, p1);
    }
    const int n = min(32, total - c);
    for (int i = 0; i < n; ++i) {
      const int ow = __shfl_sync(full, owner, i);
      const int ff = __shfl_sync(full, f, i);
      const double dd = __shfl_sync(full, dist.v, i);
      const double a0 = __shfl_sync(full, p0.v, i);
      const double a1 = __shfl_sync(full, p1.v, i);
      if (lane == ow) {
        if (ff < 9) seg.offer(xf64(dd), ff, xf64(a0), xf64(a1));
        else pt.offer(xf64(dd), ff - 9, xf64(a0), xf64(a1));
      }
    }
  }
  __syncwarp();
  // ---- 4. selection (bf.cpp:1102) and closest points --------------------------------
  if (pt.dist > seg.dist) feature_points_dyn(Ax, Bx, seg.f, seg.p0, seg.p1, pq);
  else feature_points_dyn(Ax, Bx, 9 + pt.f, pt.p0, pt.p1, pq);
  return 1 + cnt;
}

}  // namespace delta
