// tri_zoltan.cuh -- the narrowphase of the reference's zoltan/ code path in FP64
// (zoltan/bf.cpp, penalty.cpp, hybrid.cpp), written over xf64 so that every operation
// rounds once, in the reference's order.  The only operations that are not +, -, *, /,
// sqrt are the pow/log/log10 of the penalty weights (zoltan/penalty.cpp:88,
// zoltan/hybrid.cpp:166); they are CUDA's, which may differ from the host C library's in
// the last bit.
#pragma once
#include "real.cuh"
#include "tri_ref.cuh"

namespace delta {
namespace zoltan {

using X = xf64;

// zoltan/bf.cpp:26-952 for one pair (vertex v, coordinate k).  bfSolver's features and
// arithmetic with the zoltan copy's differences: early return (outputs untouched, return
// value true) on B's zero cross product (B1-B0)x(B2-B1) (zoltan/bf.cpp:68-79) or when B's
// x component and A's y, z components of (A1-A0)x(A2-A0) are zero (zoltan/bf.cpp:117-119);
// no break after case 1 of either switch (zoltan/bf.cpp:524-539, 907-914), so edge pair 1
// gets edge pair 2's point on B and vertex-face feature 1 gets B's vertex 2.
__device__ __forceinline__ bool bf_pair(const X A[3][3], const X B[3][3], X pq[6]) {
  X u[3], v[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    u[k] = B[1][k] - B[0][k];
    v[k] = B[2][k] - B[1][k];
  }
  const X nb0 = u[1] * v[2] - u[2] * v[1], nb1 = u[2] * v[0] - u[0] * v[2], nb2 = u[0] * v[1] - u[1] * v[0];
  if (nb0.v == 0.0 && nb1.v == 0.0 && nb2.v == 0.0) return true;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    u[k] = A[1][k] - A[0][k];
    v[k] = A[2][k] - A[0][k];
  }
  const X na1 = u[2] * v[0] - u[0] * v[2], na2 = u[0] * v[1] - u[1] * v[0];
  if (nb0.v == 0.0 && na1.v == 0.0 && na2.v == 0.0) return true;

  X ssmin = X(1E+30), ssc = X(0.0), ttc = X(0.0);
  int ssid = 0;
#pragma unroll
  for (int j = 0; j < 9; ++j) {
    X sc, tc;
    const X dist = seg_seg_ref(A[j / 3], A[(j / 3 + 1) % 3], B[j % 3], B[(j % 3 + 1) % 3], sc, tc);
    if (dist < ssmin) { ssmin = dist; ttc = tc; ssc = sc; ssid = j; }
  }
  X ptmin = X(1E30), ss = X(0.0), tt = X(0.0);
  int id = 0;
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    X s, t;
    const X dist = j < 3 ? pt_tri_ref(A[0], A[1], A[2], B[j], s, t) : pt_tri_ref(B[0], B[1], B[2], A[j - 3], s, t);
    if (dist < ptmin) { ptmin = dist; ss = s; tt = t; id = j; }
  }
  // the edge-edge switch always writes; case 1 continues into case 2's point on B
  {
    X pqa[6], pqb[6];
    seg_seg_points(A, B, ssid, ssc, ttc, pqa);
    seg_seg_points(A, B, ssid == 1 ? 2 : ssid, ssc, ttc, pqb);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      pq[k] = pqa[k];
      pq[3 + k] = pqb[3 + k];
    }
  }
  if (ptmin > ssmin) return false;
  if (id == 1) {  // case 1 continues into case 2: B's vertex 2
    pt_tri_points(A, B, 1, ss, tt, pq);
#pragma unroll
    for (int k = 0; k < 3; ++k) pq[3 + k] = B[2][k];
  } else {
    pt_tri_points(A, B, id, ss, tt, pq);
  }
  return false;
}

__device__ __forceinline__ void hessian(const X BA[3], const X CA[3], const X ED[3], const X FD[3], X h[16]) {
  const X two = X(2.), mtwo = X(-2.);
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
}

// The quasi-Newton step of zoltan/penalty.cpp:95-170 and zoltan/hybrid.cpp:170-249 (the
// fused symmetric elimination of penaltySolver).
__device__ __forceinline__ void newton_step(const X A[3], const X D[3], const X BA[3], const X CA[3], const X ED[3],
                                            const X FD[3], const X h[16], X r, X delta, const X x[4], X dx[4]) {
  const X zero = X(0.0), one = X(1.0), two = X(2.0), mtwo = X(-2.0);
  X dh[8], mx[6], a[16], b[4], S[3];
  const bool c0 = (-x[0] <= zero), c1 = (-x[1] <= zero), c2 = (x[0] + x[1] - one <= zero);
  const bool c3 = (-x[2] <= zero), c4 = (-x[3] <= zero), c5 = (x[2] + x[3] - one <= zero);
  dh[0] = c0 ? zero : X(-1.0); mx[0] = c0 ? zero : -x[0];
  dh[2] = c1 ? zero : X(-1.0); mx[1] = c1 ? zero : -x[1];
  dh[1] = dh[3] = c2 ? zero : one; mx[2] = c2 ? zero : x[0] + x[1] - one;
  dh[4] = c3 ? zero : X(-1.0); mx[3] = c3 ? zero : -x[2];
  dh[6] = c4 ? zero : X(-1.0); mx[4] = c4 ? zero : -x[3];
  dh[5] = dh[7] = c5 ? zero : one; mx[5] = c5 ? zero : x[2] + x[3] - one;
#pragma unroll
  for (int k = 0; k < 3; ++k)
    S[k] = (A[k] + (BA[k] * x[0]) + (CA[k] * x[1])) - (D[k] + (ED[k] * x[2]) + (FD[k] * x[3]));
  b[0] = two * dot3(S, BA) + r * (dh[0] * mx[0] + dh[1] * mx[2]);
  a[0] = h[0] + r * (dh[0] * dh[0] + dh[1] * dh[1]) + delta;
  a[4] = h[4] + r * (dh[3] * dh[1]);
  const X t1 = (h[1] + r * (dh[1] * dh[3])) / a[0];
  a[13] = h[13] - h[12] * t1;
  a[9] = h[9] - h[8] * t1;
  a[5] = (h[5] + r * (dh[2] * dh[2] + dh[3] * dh[3]) + delta) - a[4] * t1;
  b[1] = (two * dot3(S, CA) + r * (dh[2] * mx[1] + dh[3] * mx[2])) - b[0] * t1;
  const X t2 = h[2] / a[0];
  const X t3 = h[3] / a[0];
  const X t4 = ((h[6]) - a[4] * t2) / a[5];
  a[14] = ((h[14] + r * (dh[7] * dh[5])) - h[12] * t2) - a[13] * t4;
  a[10] = ((h[10] + r * (dh[4] * dh[4] + dh[5] * dh[5]) + delta) - h[8] * t2) - a[9] * t4;
  b[2] = ((mtwo * dot3(S, ED) + r * (dh[4] * mx[3] + dh[5] * mx[5])) - b[0] * t2) - b[1] * t4;
  const X t5 = (h[7] - a[4] * t3) / a[5];
  const X t6 = (((h[11] + r * (dh[5] * dh[7])) - h[8] * t3) - a[9] * t5) / a[10];
  dx[3] = ((((mtwo * dot3(S, FD) + r * (dh[6] * mx[4] + dh[7] * mx[5])) - b[2] * t6) - b[0] * t3) - b[1] * t5) /
          ((((h[15] + r * (dh[6] * dh[6] + dh[7] * dh[7]) + delta) - h[12] * t3) - a[13] * t5) - a[14] * t6);
  dx[2] = (b[2] - (a[14] * dx[3])) / a[10];
  dx[1] = (b[1] - (a[9] * dx[2] + a[13] * dx[3])) / a[5];
  dx[0] = (b[0] - (a[4] * dx[1] + h[8] * dx[2] + h[12] * dx[3])) / a[0];
}

// zoltan/penalty.cpp:36-189 for list entry i (the index enters the delta update).
__device__ __forceinline__ void penalty5(const X A[3], const X Bv[3], const X Cv[3], const X D[3], const X E[3],
                                         const X F[3], uint32_t i, X P[3], X Q[3]) {
  X BA[3], CA[3], ED[3], FD[3], h[16];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    BA[k] = Bv[k] - A[k];
    CA[k] = Cv[k] - A[k];
    ED[k] = E[k] - D[k];
    FD[k] = F[k] - D[k];
  }
  hessian(BA, CA, ED, FD, h);
  const X tr = h[0] + h[5] + h[10] + h[15];
  X delta = tr * X(0.1);
  const X lambda = sqrt_(X(0.0125) * tr);
  const X r = lambda * X(pow(10.0, (X(log(lambda.v)) + X(14.0)).v));
  X x[4] = {X(0.33), X(0.33), X(0.33), X(0.33)}, dx[4];
  for (int j = 0; j < 5; ++j) {
    delta = i < 4 ? delta : r * delta;
    newton_step(A, D, BA, CA, ED, FD, h, r, delta, x, dx);
#pragma unroll
    for (int k = 0; k < 4; ++k) x[k] = x[k] - dx[k];
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    P[k] = A[k] + (BA[k] * x[0]) + (CA[k] * x[1]);
    Q[k] = D[k] + (ED[k] * x[2]) + (FD[k] * x[3]);
  }
}

// zoltan/hybrid.cpp:134-278: 7 steps, delta = 1e-16 tr(H), r = lambda 10^(log10 lambda + 8),
// error = sqrt(|dx|^2/|x|^2) of the last step.
__device__ __forceinline__ X penalty7(const X A[3], const X Bv[3], const X Cv[3], const X D[3], const X E[3],
                                      const X F[3], X P[3], X Q[3]) {
  X BA[3], CA[3], ED[3], FD[3], h[16];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    BA[k] = Bv[k] - A[k];
    CA[k] = Cv[k] - A[k];
    ED[k] = E[k] - D[k];
    FD[k] = F[k] - D[k];
  }
  hessian(BA, CA, ED, FD, h);
  const X tr = h[0] + h[5] + h[10] + h[15];
  const X delta = tr * X(1E-16);
  const X lambda = sqrt_(X(0.0125) * tr);
  const X r = lambda * X(pow(10.0, (X(log10(lambda.v)) + X(8.0)).v));
  X x[4] = {X(0.33), X(0.33), X(0.33), X(0.33)}, dx[4];
  for (int i = 0; i < 7; ++i) {
    newton_step(A, D, BA, CA, ED, FD, h, r, delta, x, dx);
#pragma unroll
    for (int k = 0; k < 4; ++k) x[k] = x[k] - dx[k];
  }
  const X dd = (dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]) + dx[3] * dx[3];
  const X xx = (x[0] * x[0] + x[1] * x[1] + x[2] * x[2]) + x[3] * x[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    P[k] = A[k] + (BA[k] * x[0]) + (CA[k] * x[1]);
    Q[k] = D[k] + (ED[k] * x[2]) + (FD[k] * x[3]);
  }
  return sqrt_(dd / xx);
}

// segt, zoltan/hybrid.cpp:280-342 (P is written once the crossing parameter is in [0,1]).
__device__ __forceinline__ int segt(const X p1[3], const X p2[3], const X A[3], const X B[3], const X C[3], X P[3]) {
  X u[3], v[3], n[3], dir[3], w0[3], w[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    u[k] = B[k] - A[k];
    v[k] = C[k] - A[k];
  }
  n[0] = u[1] * v[2] - u[2] * v[1];
  n[1] = u[2] * v[0] - u[0] * v[2];
  n[2] = u[0] * v[1] - u[1] * v[0];
  if (n[0].v == 0.0 && n[1].v == 0.0 && n[2].v == 0.0) return -1;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    dir[k] = p2[k] - p1[k];
    w0[k] = p1[k] - A[k];
  }
  const X a = -dot3(n, w0);
  const X b = dot3(n, dir);
  if (fabs(b.v) < 1E-99 && a.v == 0.0) return 2;
  const X r = a / b;
  if (r < X(0.0) || r > X(1.0)) return 0;
#pragma unroll
  for (int k = 0; k < 3; ++k) P[k] = p1[k] + r * dir[k];
  const X uu = dot3(u, u), uv = dot3(u, v), vv = dot3(v, v);
#pragma unroll
  for (int k = 0; k < 3; ++k) w[k] = P[k] - A[k];
  const X wu = dot3(w, u), wv = dot3(w, v);
  const X Dd = uv * uv - uu * vv;
  const X s = (uv * wv - vv * wu) / Dd;
  if (s < X(0.0) || s > X(1.0)) return 0;
  const X t = (uv * wu - uu * wv) / Dd;
  if (t < X(0.0) || (s + t) > X(1.0)) return 0;
  return 1;
}

// segseg, zoltan/hybrid.cpp:344-445: SMALL_NUM = 1e-8; Q's y and z start from p4's x
// (hybrid.cpp:436-437); the distance is that of the correct points.
__device__ __forceinline__ X segseg(const X p1[3], const X p2[3], const X p3[3], const X p4[3], X P[3], X Q[3]) {
  X u[3], v[3], w[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    u[k] = p1[k] - p2[k];
    v[k] = p3[k] - p4[k];
    w[k] = p2[k] - p4[k];
  }
  const X a = dot3(u, u), b = dot3(u, v), c = dot3(v, v), d = dot3(u, w), e = dot3(v, w);
  const X Dd = a * c - b * b;
  X sD = Dd, tD = Dd, sN = X(0.0), tN = X(0.0);
  const X SMALL = X(0.00000001);
  if (Dd < SMALL) {
    sN = X(0.0); sD = X(1.0); tN = e; tD = c;
  } else {
    sN = (b * e - c * d);
    tN = (a * e - b * d);
    if (sN < X(0.0)) { sN = X(0.0); tN = e; tD = c; }
    else if (sN > sD) { sN = sD; tN = e + b; tD = c; }
  }
  const X md = -d;
  if (tN < X(0.0)) {
    tN = X(0.0);
    if (md < X(0.0)) sN = X(0.0);
    else if (md > a) sN = sD;
    else { sN = md; sD = a; }
  } else if (tN > tD) {
    tN = tD;
    const X mdb = md + b;
    if (mdb < X(0.0)) sN = X(0.0);
    else if (mdb > a) sN = sD;
    else { sN = mdb; sD = a; }
  }
  const X sc = (fabs_(sN) < SMALL) ? X(0.0) : sN / sD;
  const X tc = (fabs_(tN) < SMALL) ? X(0.0) : tN / tD;
#pragma unroll
  for (int k = 0; k < 3; ++k) P[k] = p2[k] + u[k] * sc;
  Q[0] = p4[0] + v[0] * tc;
  Q[1] = p4[0] + v[1] * tc;
  Q[2] = p4[0] + v[2] * tc;
  X dP[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) dP[k] = w[k] + (sc * u[k]) - (tc * v[k]);
  return sqrt_(dot3(dP, dP));
}

// point.cpp's pt (the zoltan/hybrid.cpp:447-644 copy is the same): closest point tq of
// triangle (T1,T2,T3) to c and its distance.
__device__ __forceinline__ X pt(const X T1[3], const X T2[3], const X T3[3], const X c[3], X tq[3]) {
  X s, t;
  const X dist = pt_tri_ref<X, false>(T1, T2, T3, c, s, t);
#pragma unroll
  for (int k = 0; k < 3; ++k) tq[k] = T1[k] + ((T3[k] - T1[k]) * t) + ((T2[k] - T1[k]) * s);
  return dist;
}

__device__ __forceinline__ void copy3(X *dst, const X *src) {
#pragma unroll
  for (int k = 0; k < 3; ++k) dst[k] = src[k];
}

// bf, zoltan/hybrid.cpp:646-886.  P and Q are in/out: a crossing found by segt gives
// Q = P; with NaN distances no branch writes them.
__device__ __forceinline__ void hybrid_bf(const X A[3], const X B[3], const X C[3], const X D[3], const X E[3],
                                          const X F[3], X P[3], X Q[3]) {
  int intersection = 0;
  if (segt(D, E, A, B, C, P) == 1) intersection = 1;
  else if (segt(E, F, A, B, C, P) == 1) intersection = 1;
  else if (segt(F, D, A, B, C, P) == 1) intersection = 1;
  else if (segt(A, B, D, E, F, P) == 1) intersection = 1;
  else if (segt(B, C, D, E, F, P) == 1) intersection = 1;
  else if (segt(C, A, D, E, F, P) == 1) intersection = 1;
  if (intersection == 1) {
    copy3(Q, P);
    return;
  }
  const X *av[3] = {A, B, C}, *bv[3] = {D, E, F};
  X tp[3], tq[3], tmpP[3], tmpQ[3], ssP[3], ssQ[3], ptmin = X(1E+30), ssmin = X(1E+30);
  for (int j = 0; j < 3; ++j) {  // A's vertices against DEF; the first is taken as is
    const X tmp = pt(D, E, F, av[j], tmpP);
    if (j == 0 || ptmin > tmp) {
      ptmin = tmp;
      copy3(tp, av[j]);
      copy3(tq, tmpP);
    }
  }
  for (int j = 0; j < 3; ++j) {  // B's vertices against ABC
    const X tmp = pt(A, B, C, bv[j], tmpP);
    if (ptmin > tmp) {
      ptmin = tmp;
      copy3(tq, bv[j]);
      copy3(tp, tmpP);
    }
  }
  for (int ea = 0; ea < 3; ++ea)
    for (int eb = 0; eb < 3; ++eb) {
      const X tmp = segseg(av[ea], av[(ea + 1) % 3], bv[eb], bv[(eb + 1) % 3], tmpP, tmpQ);
      if ((ea == 0 && eb == 0) || ssmin > tmp) {
        ssmin = tmp;
        copy3(ssP, tmpP);
        copy3(ssQ, tmpQ);
      }
    }
  if (ssmin < ptmin) {
    copy3(P, ssP);
    copy3(Q, ssQ);
  } else if (ssmin > ptmin) {
    copy3(P, tp);
    copy3(Q, tq);
  } else if (ssmin == ptmin) {
    copy3(P, ssP);
    copy3(Q, tq);
  }
}

// zoltan/dynamics.cpp:338-414 is delta/dynamics/dynamics.cpp:26-102 (expmap in pose.cuh).

}  // namespace zoltan
}  // namespace delta
