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

// Clamp to [0, 1] in the producing instruction (.sat), NaN to 0: a clamped parameter only
// has to be a feasible point of its segment or triangle for the bounds below to hold.
__device__ __forceinline__ float clamp01(float x) { return __saturatef(x); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }

// The per-triangle constants of an FP32 point-triangle projection (edges from vertex 0,
// Gram entries, the reciprocals of the four divisions), formed once per triangle for all
// the points projected onto it.
struct TriFrame {
  float e0[3], e1[3];
  float a, b, c, idet, ra, rc, rden;
};

__device__ __forceinline__ TriFrame tri_frame(const float V[3][3]) {
  TriFrame F;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    F.e0[k] = V[1][k] - V[0][k];
    F.e1[k] = V[2][k] - V[0][k];
  }
  F.a = dot3(F.e0, F.e0);
  F.b = dot3(F.e0, F.e1);
  F.c = dot3(F.e1, F.e1);
  F.idet = __fdividef(1.f, fmaf(F.a, F.c, -F.b * F.b));
  F.ra = __fdividef(1.f, F.a);
  F.rc = __fdividef(1.f, F.c);
  F.rden = __fdividef(1.f, F.a - 2.f * F.b + F.c);
  return F;
}

// The per-edge constants of the FP32 edge-edge bound: the edge from its tail to its head,
// its squared length and the reciprocal of that, formed once per edge for the three edge
// pairs it is in.
struct EdgeFrame {
  float u[3];
  float a, ra;
};

__device__ __forceinline__ EdgeFrame edge_frame(const float *H, const float *T) {
  EdgeFrame E;
#pragma unroll
  for (int k = 0; k < 3; ++k) E.u[k] = H[k] - T[k];
  E.a = dot3(E.u, E.u);
  E.ra = fdiv(1.f, E.a);
  return E;
}

// FP32 edge-edge: clamped closest parameters (segment P(s)=TA+s*u, Q(t)=TB+t*v, with u and
// v the edges of U and V), the distance of that point pair and its Frank-Wolfe lower bound.
// Returns d, writes lb.
__device__ __forceinline__ float seg_seg_lb(const float *TA, const EdgeFrame &U, const float *TB,
                                            const EdgeFrame &V, float &lb) {
  const float *u = U.u, *v = V.u;
  float w[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) w[k] = TA[k] - TB[k];
  const float a = U.a, e = V.a, b = dot3(u, v), c = dot3(u, w), f = dot3(v, w);
  const float den = fmaf(a, e, -b * b);
  float s = den > 1e-12f * (a * e) ? clamp01(fdiv(fmaf(b, f, -c * e), den)) : 0.f;
  const float traw = e > 0.f ? fmaf(b, s, f) * V.ra : 0.f;
  const float t = clamp01(traw);
  const float s2 = clamp01(fmaf(b, t, -c) * U.ra);  // a = 0: u = 0, c = 0, 0 * inf -> 0
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
__device__ __forceinline__ float pt_tri_lb(const float *V0, const TriFrame &F, const float *X, float eps, float &lb) {
  const float *E0 = F.e0, *E1 = F.e1;
  float D[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) D[k] = V0[k] - X[k];
  const float a = F.a, b = F.b, c = F.c, d = dot3(E0, D), e = dot3(E1, D), f = dot3(D, D);
  const float si = fmaf(b, e, -c * d) * F.idet, ti = fmaf(b, d, -a * e) * F.idet;
  const bool inside = si >= 0.f && ti >= 0.f && si + ti <= 1.f;
  // squared distance of parameter (s,t) less f: |D + s E0 + t E1|^2 - f
  //   = 2(s d + t e) + s^2 a + 2 s t b + t^2 c (it only ranks the three edge points)
  auto q = [&](float s, float t) { return fmaf(s, fmaf(a, s, fmaf(2.f * b, t, 2.f * d)), t * fmaf(c, t, 2.f * e)); };
  // degenerate edges give 0/0, which clamp01 sends to 0; any value in [0, 1] is feasible
  const float s0 = clamp01(-d * F.ra);  // edge t = 0
  const float t1 = clamp01(-e * F.rc);  // edge s = 0
  const float l2 = clamp01((c + e - b - d) * F.rden);  // edge s + t = 1: s = l2
  float s = s0, t = 0.f, best = s0 * fmaf(a, s0, 2.f * d);  // q(s0, 0)
  const float q1 = t1 * fmaf(c, t1, 2.f * e), q2 = q(l2, 1.f - l2);  // q(0, t1), q(l2, 1 - l2)
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

// Per-warp shared staging for bf_cert_warp: the 32 pairs' FP64 coordinates, the
// candidate queues (one per feature family) and the queue results.
constexpr int kCertQueue = 64;  // entries evaluated per pass and family
struct CertWarpSmem {
  double coords[32][18];
  uint8_t qs[32 * 9], qp[32 * 6];      // queued (lane << 0) with features in a separate array
  uint8_t fs[32 * 9], fp[32 * 6];
  double rd[kCertQueue], r0[kCertQueue], r1[kCertQueue];
  int32_t surv[64];  // particle-pair driver: B triangles that passed the box test
};

// Running minimum of one feature family, ordered by (distance, feature index): equal to
// the reference's sequential scan with strict < (first minimum wins).
struct FamilyBest {
  xf64 dist, p0, p1;
  int f;
  __device__ __forceinline__ void offer(xf64 d, int ff, xf64 a, xf64 b) {
    if (d < dist || (d == dist && ff < f)) { dist = d; f = ff; p0 = a; p1 = b; }
  }
};

__device__ __forceinline__ void load_pair(const CertWarpSmem &sm, int lane, xf64 A[3][3], xf64 B[3][3]) {
#pragma unroll
  for (int v = 0; v < 3; ++v)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      A[v][k] = xf64(sm.coords[lane][3 * v + k]);
      B[v][k] = xf64(sm.coords[lane][9 + 3 * v + k]);
    }
}

// Edge-edge feature f (0..8) of the pair staged for `lane`.
__device__ __forceinline__ xf64 seg_dyn(const CertWarpSmem &sm, int lane, int f, xf64 &p0, xf64 &p1) {
  const int ea = f / 3, eb = f - 3 * ea;
  const int ta = ea == 2 ? 0 : ea + 1, tb = eb == 2 ? 0 : eb + 1;
  xf64 HA[3], TA[3], HB[3], TB[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    HA[k] = xf64(sm.coords[lane][3 * ea + k]);
    TA[k] = xf64(sm.coords[lane][3 * ta + k]);
    HB[k] = xf64(sm.coords[lane][9 + 3 * eb + k]);
    TB[k] = xf64(sm.coords[lane][9 + 3 * tb + k]);
  }
  return seg_seg_ref(HA, TA, HB, TB, p0, p1);
}

// Vertex-face feature j (0..5) of the pair staged for `lane`.
__device__ __forceinline__ xf64 pt_dyn(const CertWarpSmem &sm, int lane, int j, xf64 &p0, xf64 &p1) {
  const int tri = j < 3 ? 0 : 9, pnt = j < 3 ? 9 + 3 * j : 3 * (j - 3);
  xf64 V0[3], V1[3], V2[3], X[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    V0[k] = xf64(sm.coords[lane][tri + k]);
    V1[k] = xf64(sm.coords[lane][tri + 3 + k]);
    V2[k] = xf64(sm.coords[lane][tri + 6 + k]);
    X[k] = xf64(sm.coords[lane][pnt + k]);
  }
  return pt_tri_ref(V0, V1, V2, X, p0, p1);
}

// Evaluates a family's queue (entries: lane, feature) in passes of kCertQueue and offers
// each result to its owner's running minimum.  owner_lo/owner_cnt: this lane's entries.
template <bool SEG>
__device__ __forceinline__ void run_queue(CertWarpSmem &sm, const uint8_t *ql, const uint8_t *qf, int total,
                                          int my_lo, int my_cnt, FamilyBest &best) {
  const int lane = threadIdx.x & 31;
  for (int base = 0; base < total; base += kCertQueue) {
    const int n = min(kCertQueue, total - base);
    for (int j = lane; j < n; j += 32) {
      xf64 p0, p1;
      const xf64 d = SEG ? seg_dyn(sm, ql[base + j], qf[base + j], p0, p1) : pt_dyn(sm, ql[base + j], qf[base + j], p0, p1);
      sm.rd[j] = d.v;
      sm.r0[j] = p0.v;
      sm.r1[j] = p1.v;
    }
    __syncwarp();
    const int lo = max(my_lo, base), hi = min(my_lo + my_cnt, base + n);
    for (int j = lo; j < hi; ++j)
      best.offer(xf64(sm.rd[j - base]), qf[j], xf64(sm.r0[j - base]), xf64(sm.r1[j - base]));
    __syncwarp();
  }
}

__device__ __forceinline__ int warp_excl_scan(int v, int &total) {
  const int lane = threadIdx.x & 31;
  int incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  total = __shfl_sync(0xffffffffu, incl, 31);
  return incl - v;
}

// All 32 lanes call this together; lanes with valid == false carry dummy data and
// produce nothing.  Writes bfSolver's closest points to pq; returns the number of FP64
// feature evaluations made for this lane's pair.
__device__ __forceinline__ int bf_cert_warp(const double A64[3][3], const double B64[3][3], bool valid, double pq[6],
                                            CertWarpSmem &sm) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int v = 0; v < 3; ++v)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      sm.coords[lane][3 * v + k] = A64[v][k];
      sm.coords[lane][9 + 3 * v + k] = B64[v][k];
    }
  // ---- 1. FP32 lower bounds -------------------------------------------------------
  float A[3][3], B[3][3];
  double L = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double lo = A64[0][k], hi = A64[0][k];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      A[v][k] = v == 0 ? 0.f : (float)(A64[v][k] - A64[0][k]);  // A's vertex 0 is the origin
      B[v][k] = (float)(B64[v][k] - A64[0][k]);
      lo = fmin(lo, fmin(A64[v][k], B64[v][k]));
      hi = fmax(hi, fmax(A64[v][k], B64[v][k]));
    }
    L = fmax(L, hi - lo);
  }
  const float eps = (float)L * (64.f * kU32);
  float lb[15];
  int sbest = 0, pbest = 0;
  float sd = 3.0e38f, pd = 3.0e38f;
  {
    // edge j of a triangle runs from vertex j+1 (tail) to vertex j (head); each edge is
    // in three edge pairs
    EdgeFrame EA[3], EB[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      EA[j] = edge_frame(A[j], A[(j + 1) % 3]);
      EB[j] = edge_frame(B[j], B[(j + 1) % 3]);
    }
#pragma unroll
    for (int j = 0; j < 9; ++j) {
      float l;
      const float d = seg_seg_lb(A[(j / 3 + 1) % 3], EA[j / 3], B[(j % 3 + 1) % 3], EB[j % 3], l);
      lb[j] = l - eps;
      if (d < sd) { sd = d; sbest = j; }
    }
  }
  {
    const TriFrame FA = tri_frame(A), FB = tri_frame(B);
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      float d = pt_tri_lb(A[0], FA, B[j], eps, lb[9 + j]);
      if (d < pd) { pd = d; pbest = j; }
      d = pt_tri_lb(B[0], FB, A[j], eps, lb[12 + j]);
      if (d < pd) { pd = d; pbest = 3 + j; }
    }
  }
  __syncwarp();
  // ---- 2. FP64 values of each family's FP32 argmin (every lane runs both paths) --------
  FamilyBest seg{xf64(1E+30), xf64(0.0), xf64(0.0), 0}, pt{xf64(1E30), xf64(0.0), xf64(0.0), 0};
  {
    xf64 a0, a1;
    const xf64 ds = seg_dyn(sm, lane, sbest, a0, a1);
    if (ds < seg.dist) { seg.dist = ds; seg.f = sbest; seg.p0 = a0; seg.p1 = a1; }
    const xf64 dp = pt_dyn(sm, lane, pbest, a0, a1);
    if (dp < pt.dist) { pt.dist = dp; pt.f = pbest; pt.p0 = a0; pt.p1 = a1; }
  }
  const double best = fmin(seg.dist.v, pt.dist.v);  // NaN-free unless both are NaN
  const double bound = (best == best) ? best : 1.0e308;
  // ---- 3. queue the remaining candidates, one queue per family ------------------------
  unsigned ms = 0, mp = 0;
#pragma unroll
  for (int f = 0; f < 9; ++f)
    if (f != sbest && !((double)lb[f] > bound)) ms |= 1u << f;
#pragma unroll
  for (int j = 0; j < 6; ++j)
    if (j != pbest && !((double)lb[9 + j] > bound)) mp |= 1u << j;
  if (!valid) ms = mp = 0;
  int ts, tp;
  const int cs = __popc(ms), cp = __popc(mp);
  const int os = warp_excl_scan(cs, ts), op = warp_excl_scan(cp, tp);
  {
    int q = os;
    for (unsigned m = ms; m; m &= m - 1) { sm.qs[q] = (uint8_t)lane; sm.fs[q] = (uint8_t)(__ffs(m) - 1); ++q; }
    q = op;
    for (unsigned m = mp; m; m &= m - 1) { sm.qp[q] = (uint8_t)lane; sm.fp[q] = (uint8_t)(__ffs(m) - 1); ++q; }
  }
  __syncwarp();
  run_queue<true>(sm, sm.qs, sm.fs, ts, os, cs, seg);
  run_queue<false>(sm, sm.qp, sm.fp, tp, op, cp, pt);
  // ---- 4. selection (bf.cpp:1102) and closest points --------------------------------
  xf64 Ax[3][3], Bx[3][3];
  load_pair(sm, lane, Ax, Bx);
  __syncwarp();
  if (pt.dist > seg.dist) feature_points_dyn(Ax, Bx, seg.f, seg.p0, seg.p1, pq);
  else feature_points_dyn(Ax, Bx, 9 + pt.f, pt.p0, pt.p1, pq);
  return 2 + cs + cp;
}

}  // namespace delta
