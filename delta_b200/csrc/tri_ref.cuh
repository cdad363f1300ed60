// tri_ref.cuh -- triangle-triangle narrowphase with the reference's arithmetic.
//
// Templated over the arithmetic type R (xf64 for the FP64 path, float for FP32).  Each
// routine performs the same rounded operations, in the same order, as the reference
// function it cites, so that R = xf64 reproduces the reference bit for bit.  A triangle
// is R T[3][3] (vertex, coordinate).
#pragma once
#include "real.cuh"

namespace delta {

// Closest points of edge (HA<-TA) and edge (HB<-TB): Sunday's clamped parameters as
// written in bf.cpp:586-697.  The edge runs from its tail T (parameter 0) to its head H
// (parameter 1).  Returns |dP|^2 (seg_seg_ref: |dP|).
template <class R>
__device__ __forceinline__ R seg_seg_sq_ref(const R *HA, const R *TA, const R *HB, const R *TB, R &sc, R &tc) {
  R u[3], v[3], w[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    u[k] = HA[k] - TA[k];
    v[k] = HB[k] - TB[k];
    w[k] = TA[k] - TB[k];
  }
  const R a = dot3(u, u), b = dot3(u, v), c = dot3(v, v), d = dot3(u, w), e = dot3(v, w);
  const R D = a * c - b * b;
  const R SMALL = R(1e-30);
  R sD = D, tD = D, sN, tN;
  if (D < SMALL) {
    sN = R(0.0); sD = R(1.0); tN = e; tD = c;
  } else {
    sN = b * e - c * d;
    tN = a * e - b * d;
    if (sN < R(0.0)) { sN = R(0.0); tN = e; tD = c; }
    else if (sN > sD) { sN = sD; tN = e + b; tD = c; }
  }
  const R md = -d;
  if (tN < R(0.0)) {
    tN = R(0.0);
    if (md < R(0.0)) sN = R(0.0);
    else if (md > a) sN = sD;
    else { sN = md; sD = a; }
  } else if (tN > tD) {
    tN = tD;
    const R mdb = md + b;
    if (mdb < R(0.0)) sN = R(0.0);
    else if (mdb > a) sN = sD;
    else { sN = mdb; sD = a; }
  }
  sc = (fabs_(sN) < SMALL) ? R(0.0) : sN / sD;
  tc = (fabs_(tN) < SMALL) ? R(0.0) : tN / tD;
  R dP[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) dP[k] = (TA[k] - TB[k]) + (sc * (HA[k] - TA[k])) - (tc * (HB[k] - TB[k]));
  return dP[0] * dP[0] + dP[1] * dP[1] + dP[2] * dP[2];
}

template <class R>
__device__ __forceinline__ R seg_seg_ref(const R *HA, const R *TA, const R *HB, const R *TB, R &sc, R &tc) {
  return sqrt_(seg_seg_sq_ref(HA, TA, HB, TB, sc, tc));
}

// Point X against triangle (V0,V1,V2): Eberly's seven regions as written in
// bf.cpp:920-1090.  s runs along V1-V0, t along V2-V0.  Returns the clamped squared
// distance (pt_tri_ref: the distance).  The final clamp of the squared distance is
// bf.cpp:1090's `<= 0` (kClampLE) or point.cpp:199's and zoltan/hybrid.cpp's `< 0`; they
// differ only for -0.0, which `<` keeps.
template <class R, bool kClampLE = true>
__device__ __forceinline__ R pt_tri_sq_ref(const R *V0, const R *V1, const R *V2, const R *X, R &s_out, R &t_out) {
  R E0[3], E1[3], Dv[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    E0[k] = V1[k] - V0[k];
    E1[k] = V2[k] - V0[k];
    Dv[k] = V0[k] - X[k];
  }
  const R a = dot3(E0, E0), b = dot3(E0, E1), c = dot3(E1, E1);
  const R d = dot3(E0, Dv), e = dot3(E1, Dv), f = dot3(Dv, Dv);
  const R det = a * c - b * b;
  R s = b * e - c * d;
  R t = b * d - a * e;
  R sq;
  const R zero = R(0), one = R(1), two = R(2);
  // the interior formula s*(a s + b t + 2d) + t*(b s + c t + 2e) + f
#define DELTA_FULLQ (s * (a * s + b * t + two * d) + t * (b * s + c * t + two * e) + f)
  if ((s + t) <= det) {
    if (s < zero) {
      if (t < zero) {  // region 4
        if (d < zero) {
          t = zero;
          if (-d >= a) { s = one; sq = a + two * d + f; }
          else { s = -d / a; sq = d * s + f; }
        } else {
          s = zero;
          if (e >= zero) { t = zero; sq = f; }
          else if (-e >= c) { t = one; sq = c + two * e + f; }
          else { t = -e / c; sq = e * t + f; }
        }
      } else {  // region 3
        s = zero;
        if (e >= zero) { t = zero; sq = f; }
        else if (-e >= c) { t = one; sq = c + two * e + f; }
        else { t = -e / c; sq = e * t + f; }
      }
    } else if (t < zero) {  // region 5
      t = zero;
      if (d >= zero) { s = zero; sq = f; }
      else if (-d >= a) { s = one; sq = a + two * d + f; }
      else { s = -d / a; sq = d * s + f; }
    } else {  // region 0
      const R inv = one / det;
      s = s * inv;
      t = t * inv;
      sq = DELTA_FULLQ;
    }
  } else {
    if (s < zero) {  // region 2
      const R tmp0 = b + d, tmp1 = c + e;
      if (tmp1 > tmp0) {
        const R numer = tmp1 - tmp0, denom = a - two * b + c;
        if (numer >= denom) { s = one; t = zero; sq = a + two * d + f; }
        else { s = numer / denom; t = one - s; sq = DELTA_FULLQ; }
      } else {
        s = zero;
        if (tmp1 <= zero) { t = one; sq = c + two * e + f; }
        else if (e >= zero) { t = zero; sq = f; }
        else { t = -e / c; sq = e * t + f; }
      }
    } else if (t < zero) {  // region 6
      const R tmp0 = b + e, tmp1 = a + d;
      if (tmp1 > tmp0) {
        const R numer = tmp1 - tmp0, denom = a - two * b + c;
        if (numer >= denom) { t = one; s = zero; sq = c + two * e + f; }
        else { t = numer / denom; s = one - t; sq = DELTA_FULLQ; }
      } else {
        t = zero;
        if (tmp1 <= zero) { s = one; sq = a + two * d + f; }
        else if (d >= zero) { s = zero; sq = f; }
        else { s = -d / a; sq = d * s + f; }
      }
    } else {  // region 1
      const R numer = c + e - b - d;
      if (numer <= zero) { s = zero; t = one; sq = c + two * e + f; }
      else {
        const R denom = a - two * b + c;
        if (numer >= denom) { s = one; t = zero; sq = a + two * d + f; }
        else { s = numer / denom; t = one - s; sq = DELTA_FULLQ; }
      }
    }
  }
#undef DELTA_FULLQ
  if (kClampLE ? (sq <= zero) : (sq < zero)) sq = zero;
  s_out = s;
  t_out = t;
  return sq;
}

template <class R, bool kClampLE = true>
__device__ __forceinline__ R pt_tri_ref(const R *V0, const R *V1, const R *V2, const R *X, R &s_out, R &t_out) {
  return sqrt_(pt_tri_sq_ref<R, kClampLE>(V0, V1, V2, X, s_out, t_out));
}

// Closest point on edge pair j = 3*ea + eb for parameters (sc, tc); bf.cpp:715-879.
template <class R>
__device__ __forceinline__ void seg_seg_points(const R A[3][3], const R B[3][3], int j, R sc, R tc, R pq[6]) {
#pragma unroll
  for (int jj = 0; jj < 9; ++jj) {
    if (jj == j) {
      const int ea = jj / 3, eb = jj % 3;
      const R *HA = A[ea], *TA = A[(ea + 1) % 3], *HB = B[eb], *TB = B[(eb + 1) % 3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        pq[k] = TA[k] + ((HA[k] - TA[k]) * sc);
        pq[3 + k] = TB[k] + ((HB[k] - TB[k]) * tc);
      }
    }
  }
}

// Closest points of vertex-face feature j (0..2: B's vertex j on A; 3..5: A's vertex
// j-3 on B) for parameters (s, t); bf.cpp:1104-1177.
template <class R>
__device__ __forceinline__ void pt_tri_points(const R A[3][3], const R B[3][3], int j, R s, R t, R pq[6]) {
  const bool onA = j < 3;
  const R(*T)[3] = onA ? A : B;
  R face[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) face[k] = T[0][k] + ((T[2][k] - T[0][k]) * t) + ((T[1][k] - T[0][k]) * s);
  R vert[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    vert[k] = (j == 0 || j == 3) ? (onA ? B[0][k] : A[0][k])
            : (j == 1 || j == 4) ? (onA ? B[1][k] : A[1][k])
                                 : (onA ? B[2][k] : A[2][k]);
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    pq[k] = onA ? face[k] : vert[k];
    pq[3 + k] = onA ? vert[k] : face[k];
  }
}

// Feature f in 0..14: 0..8 edge-edge, 9..14 vertex-face.  Distance and parameters.
template <class R>
__device__ __forceinline__ R feature_ref(const R A[3][3], const R B[3][3], int f, R &p0, R &p1) {
  R dist = R(0);
#pragma unroll
  for (int j = 0; j < 9; ++j)
    if (f == j) dist = seg_seg_ref(A[j / 3], A[(j / 3 + 1) % 3], B[j % 3], B[(j % 3 + 1) % 3], p0, p1);
#pragma unroll
  for (int j = 0; j < 3; ++j)
    if (f == 9 + j) dist = pt_tri_ref(A[0], A[1], A[2], B[j], p0, p1);
#pragma unroll
  for (int j = 0; j < 3; ++j)
    if (f == 12 + j) dist = pt_tri_ref(B[0], B[1], B[2], A[j], p0, p1);
  return dist;
}

// bfSolver, bf.cpp:217-1178.  First minimum wins inside each family; the edge-edge
// result is kept only when it is strictly closer (bf.cpp:1102).
template <class R>
__device__ __forceinline__ void bf_solve_ref(const R A[3][3], const R B[3][3], R pq[6]) {
  R ssmin = R(1E+30), ssc = R(0), ttc = R(0);
  int ssid = 0;
#pragma unroll
  for (int j = 0; j < 9; ++j) {
    R sc, tc;
    const R dist = seg_seg_ref(A[j / 3], A[(j / 3 + 1) % 3], B[j % 3], B[(j % 3 + 1) % 3], sc, tc);
    if (dist < ssmin) { ssmin = dist; ttc = tc; ssc = sc; ssid = j; }
  }
  R ptmin = R(1E30), ss = R(0), tt = R(0);
  int id = 0;
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    R s, t;
    const R dist = j < 3 ? pt_tri_ref(A[0], A[1], A[2], B[j], s, t) : pt_tri_ref(B[0], B[1], B[2], A[j - 3], s, t);
    if (dist < ptmin) { ptmin = dist; ss = s; tt = t; id = j; }
  }
  if (ptmin > ssmin) seg_seg_points(A, B, ssid, ssc, ttc, pq);
  else pt_tri_points(A, B, id, ss, tt, pq);
}

// bfSolver as bf_solve_ref (the same 15 evaluations, comparisons and results), written
// for a small register footprint: the edge pairs and the vertex-face pairs run as rolled
// loops over local copies of the triangles whose vertices rotate one place per iteration,
// so one copy of each feature routine is live at a time.  Edge pair j = 3*ea + eb runs
// from U[1] to U[0] and from V[1] to V[0] after ea rotations of U and eb of V; vertex-face
// pair j < 3 tests V[0] = B[j] against U = A, and j >= 3 (U and V swapped) A[j-3] against B.
template <class R>
__device__ __forceinline__ void rotate3(R T[3][3]) {
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const R t = T[0][k];
    T[0][k] = T[1][k];
    T[1][k] = T[2][k];
    T[2][k] = t;
  }
}

template <class R>
__device__ __forceinline__ void bf_solve_lean(const R A[3][3], const R B[3][3], R pq[6]) {
  R U[3][3], V[3][3];
#pragma unroll
  for (int v = 0; v < 3; ++v)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      U[v][k] = A[v][k];
      V[v][k] = B[v][k];
    }
  R ssmin = R(1E+30), ssc = R(0), ttc = R(0);
  int ssid = 0;
#pragma unroll 1
  for (int ea = 0; ea < 3; ++ea) {
#pragma unroll 1
    for (int eb = 0; eb < 3; ++eb) {
      R sc, tc;
      const R dist = seg_seg_ref(U[0], U[1], V[0], V[1], sc, tc);
      if (dist < ssmin) { ssmin = dist; ttc = tc; ssc = sc; ssid = 3 * ea + eb; }
      rotate3(V);
    }
    rotate3(U);
  }
  R ptmin = R(1E30), ss = R(0), tt = R(0);
  int id = 0;
#pragma unroll 1
  for (int j = 0; j < 6; ++j) {
    if (j == 3) {
#pragma unroll
      for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const R t = U[v][k];
          U[v][k] = V[v][k];
          V[v][k] = t;
        }
    }
    R s, t;
    const R dist = pt_tri_ref(U[0], U[1], U[2], V[0], s, t);
    if (dist < ptmin) { ptmin = dist; ss = s; tt = t; id = j; }
    rotate3(V);
  }
  // here V = A and U = B again (A and B need not stay live through the loops)
  if (ptmin > ssmin) seg_seg_points(V, U, ssid, ssc, ttc, pq);
  else pt_tri_points(V, U, id, ss, tt, pq);
}

// penaltySolver, penalty.cpp:278-432 (adaptive = false: 4 iterations, flag = failed of
// the last step) and penalty.cpp:434-582 (adaptive = true: at most 16 iterations,
// flag = iteration index of the early exit, unchanged otherwise).
template <class R>
__device__ __forceinline__ void penalty_ref_from(const R A[3][3], const R B[3][3], R max_error, bool adaptive,
                                                 R pq[6], int &flag, const R *start) {
  R BA[3], CA[3], ED[3], FD[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    BA[k] = A[1][k] - A[0][k];
    CA[k] = A[2][k] - A[0][k];
    ED[k] = B[1][k] - B[0][k];
    FD[k] = B[2][k] - B[0][k];
  }
  const R two = R(2.), mtwo = R(-2.), zero = R(0.0), one = R(1);
  R h[16];
  h[0] = two * dot3(BA, BA);
  h[1] = two * dot3(CA, BA);
  h[2] = mtwo * dot3(ED, BA);
  h[3] = mtwo * dot3(FD, BA);
  h[4] = h[1];
  h[5] = two * dot3(CA, CA);
  h[6] = mtwo * dot3(ED, CA);
  h[7] = mtwo * dot3(FD, CA);
  h[8] = h[2];
  h[9] = h[6];
  h[10] = two * dot3(ED, ED);
  h[11] = two * dot3(FD, ED);
  h[12] = h[3];
  h[13] = h[7];
  h[14] = h[11];
  h[15] = two * dot3(FD, FD);
  R delta = (h[0] + h[5] + h[10] + h[15]) * R(1E-2);
  const R lambda = sqrt_(R(0.0125) * (h[0] + h[5] + h[10] + h[15]));
  const R r = lambda * R(1E5);
  R x[4] = {R(0.33), R(0.33), R(0.33), R(0.33)};  // initial guess, penalty.cpp:353-356
  if (start) {
    x[0] = start[0];
    x[1] = start[1];
    x[2] = start[2];
    x[3] = start[3];
  }
  const int n_iter = adaptive ? 16 : 4;
  if (!adaptive) flag = 0;
  for (int i = 0; i < n_iter; ++i) {
    R dh[8], mx[6], dx[4], a[16], b[4], S[3];
    const bool c0 = (-x[0] <= zero), c1 = (-x[1] <= zero), c2 = (x[0] + x[1] - one <= zero);
    const bool c3 = (-x[2] <= zero), c4 = (-x[3] <= zero), c5 = (x[2] + x[3] - one <= zero);
    dh[0] = c0 ? zero : R(-1); mx[0] = c0 ? zero : -x[0];
    dh[2] = c1 ? zero : R(-1); mx[1] = c1 ? zero : -x[1];
    dh[1] = dh[3] = c2 ? zero : one; mx[2] = c2 ? zero : x[0] + x[1] - one;
    dh[4] = c3 ? zero : R(-1); mx[3] = c3 ? zero : -x[2];
    dh[6] = c4 ? zero : R(-1); mx[4] = c4 ? zero : -x[3];
    dh[5] = dh[7] = c5 ? zero : one; mx[5] = c5 ? zero : x[2] + x[3] - one;
    if (adaptive) delta = i < 3 ? delta : R(1E5) * delta;
#pragma unroll
    for (int k = 0; k < 3; ++k)
      S[k] = (A[0][k] + (BA[k] * x[0]) + (CA[k] * x[1])) - (B[0][k] + (ED[k] * x[2]) + (FD[k] * x[3]));
    b[0] = two * dot3(S, BA) + r * (dh[0] * mx[0] + dh[1] * mx[2]);
    a[0] = h[0] + r * (dh[0] * dh[0] + dh[1] * dh[1]) + delta;
    a[4] = h[4] + r * (dh[3] * dh[1]);
    const R t1 = (h[1] + r * (dh[1] * dh[3])) / a[0];
    a[13] = h[13] - h[12] * t1;
    a[9] = h[9] - h[8] * t1;
    a[5] = (h[5] + r * (dh[2] * dh[2] + dh[3] * dh[3]) + delta) - a[4] * t1;
    b[1] = (two * dot3(S, CA) + r * (dh[2] * mx[1] + dh[3] * mx[2])) - b[0] * t1;
    const R t2 = h[2] / a[0];
    const R t3 = h[3] / a[0];
    const R t4 = ((h[6]) - a[4] * t2) / a[5];
    a[14] = ((h[14] + r * (dh[7] * dh[5])) - h[12] * t2) - a[13] * t4;
    a[10] = ((h[10] + r * (dh[4] * dh[4] + dh[5] * dh[5]) + delta) - h[8] * t2) - a[9] * t4;
    b[2] = ((mtwo * dot3(S, ED) + r * (dh[4] * mx[3] + dh[5] * mx[5])) - b[0] * t2) - b[1] * t4;
    const R t5 = (h[7] - a[4] * t3) / a[5];
    const R t6 = (((h[11] + r * (dh[5] * dh[7])) - h[8] * t3) - a[9] * t5) / a[10];
    dx[3] = ((((mtwo * dot3(S, FD) + r * (dh[6] * mx[4] + dh[7] * mx[5])) - b[2] * t6) - b[0] * t3) - b[1] * t5) /
            ((((h[15] + r * (dh[6] * dh[6] + dh[7] * dh[7]) + delta) - h[12] * t3) - a[13] * t5) - a[14] * t6);
    dx[2] = (b[2] - (a[14] * dx[3])) / a[10];
    dx[1] = (b[1] - (a[9] * dx[2] + a[13] * dx[3])) / a[5];
    dx[0] = (b[0] - (a[4] * dx[1] + h[8] * dx[2] + h[12] * dx[3])) / a[0];
    const R dxx = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2] + dx[3] * dx[3];
    const R xx = x[0] * x[0] + x[1] * x[1] + x[2] * x[2] + x[3] * x[3];
    if (adaptive) {
      if (dxx / xx < max_error * max_error) { flag = i; break; }
    } else {
      delta = R(1E4) * delta;
      flag = (dxx / xx > max_error * max_error) ? 1 : 0;
    }
    x[0] = x[0] - dx[0];
    x[1] = x[1] - dx[1];
    x[2] = x[2] - dx[2];
    x[3] = x[3] - dx[3];
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    pq[k] = A[0][k] + (BA[k] * x[0]) + (CA[k] * x[1]);
    pq[3 + k] = B[0][k] + (ED[k] * x[2]) + (FD[k] * x[3]);
  }
}

template <class R>
__device__ __forceinline__ void penalty_ref(const R A[3][3], const R B[3][3], R max_error, bool adaptive, R pq[6],
                                            int &flag) {
  penalty_ref_from<R>(A, B, max_error, adaptive, pq, flag, nullptr);
}

// d = |P_B - P_A| as the drivers compute it (bf.cpp:117).
template <class R>
__device__ __forceinline__ R pq_distance(const R pq[6]) {
  return sqrt_(((pq[3] - pq[0]) * (pq[3] - pq[0])) + ((pq[4] - pq[1]) * (pq[4] - pq[1])) +
               ((pq[5] - pq[2]) * (pq[5] - pq[2])));
}

}  // namespace delta
