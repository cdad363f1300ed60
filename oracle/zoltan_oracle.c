/*
 * zoltan_oracle.c -- CPU restatement (FP64) of the reference's zoltan/ code path: the
 * narrowphase functions with the SoA "one triangle against a list" shape
 * (zoltan/bf.cpp, penalty.cpp, hybrid.cpp), the contact forces (zoltan/forces.cpp) and
 * the integration (zoltan/dynamics.cpp).
 *
 * TEST INFRASTRUCTURE ONLY (the checker); see delta_oracle.h.  Compiled with
 * -ffp-contract=off: every a*b+c stays two rounded operations, in the reference's order.
 * Reference paths are relative to the project root.
 *
 * Layouts (planar, as the reference's pointer arrays `iREAL *d[3]`): d, e, f, p, q hold 3
 * planes of ld doubles, plane k = coordinate k, entry i = triangle i of the list.
 * Per-body vectors: plane k of nb doubles.  Triangles t[6][3]: plane 3*v + k of ldt
 * doubles (v = 0..2 spatial vertices, 3..5 referential vertices).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "delta_oracle.h"
#include "oracle_internal.h"

static inline double dot3z(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* The penalty weight r of list entry i moved by `ulps` units in the last place (0: as
 * computed; 1000 and above: a seeded pseudo-random shift in [-3, 3] per entry).  The
 * reference forms r with pow and log/log10, whose last bit depends on the math library;
 * the shifted variants let a test tell which results depend on that bit. */
static double shift_ulps_at(double r, int32_t ulps, uint32_t i) {
  if (ulps >= 1000) { /* a pseudo-random shift in [-3, 3] per list entry, seeded by ulps */
    uint32_t h = (i + 0x9e3779b9u * (uint32_t)ulps) ^ 0x85ebca6bu;
    h ^= h >> 15;
    h *= 0x2c1b3c6du;
    h ^= h >> 12;
    h *= 0x297a2d39u;
    h ^= h >> 15;
    ulps = (int32_t)(h % 7u) - 3;
  }
  for (; ulps > 0; --ulps) r = nextafter(r, INFINITY);
  for (; ulps < 0; ++ulps) r = nextafter(r, -INFINITY);
  return r;
}

/* ============================================================================
 * zoltan/bf.cpp:26-952, bf(xA,yA,zA, xB,yB,zB, xPA,...,zPB) for one triangle pair.
 *
 * bfSolver's features and arithmetic (bf.cpp:217-1178 of delta/contact/detection) with
 * the zoltan copy's differences kept:
 *  - early return, outputs untouched, when B's cross product (B1-B0)x(B2-B1) is zero
 *    (zoltan/bf.cpp:68-79), or when B's x component and A's y, z components of
 *    (A1-A0)x(A2-A0) are zero (the test at zoltan/bf.cpp:117-119 mixes the two normals);
 *  - the edge-edge switch has no break after case 1 (zoltan/bf.cpp:524-539): feature 1
 *    gets feature 2's point on B, p4 + (p6 - p4)*tc;
 *  - the vertex-face switch has no break after case 1 (zoltan/bf.cpp:907-914): feature 1
 *    gets B's vertex 2 instead of vertex 1.
 * The segment-triangle loop (zoltan/bf.cpp:144-191) writes the outputs from an
 * uninitialised array; the edge-edge switch always overwrites them, so it has no effect.
 * The vertex-face clamp is `< 0` here (bf.cpp's is `<= 0`); the two differ only for a
 * squared distance of -0.0, whose square root compares equal to 0.0, so the selected
 * feature and the outputs are the same.
 * Returns 1 on the early return, else 0.
 * ========================================================================== */
int dzo_bf(const double *xA, const double *yA, const double *zA, const double *xB, const double *yB,
           const double *zB, double pq[6]) {
  double u[3], v[3];
  u[0] = xB[1] - xB[0]; u[1] = yB[1] - yB[0]; u[2] = zB[1] - zB[0];
  v[0] = xB[2] - xB[1]; v[1] = yB[2] - yB[1]; v[2] = zB[2] - zB[1];
  const double nb0 = u[1] * v[2] - u[2] * v[1];
  const double nb1 = u[2] * v[0] - u[0] * v[2];
  const double nb2 = u[0] * v[1] - u[1] * v[0];
  if (nb0 == 0 && nb1 == 0 && nb2 == 0) return 1;
  u[0] = xA[1] - xA[0]; u[1] = yA[1] - yA[0]; u[2] = zA[1] - zA[0];
  v[0] = xA[2] - xA[0]; v[1] = yA[2] - yA[0]; v[2] = zA[2] - zA[0];
  const double na1 = u[2] * v[0] - u[0] * v[2];
  const double na2 = u[0] * v[1] - u[1] * v[0];
  if (nb0 == 0 && na1 == 0 && na2 == 0) return 1;

  double A[3][3], B[3][3];
  for (int w = 0; w < 3; ++w) {
    A[w][0] = xA[w]; A[w][1] = yA[w]; A[w][2] = zA[w];
    B[w][0] = xB[w]; B[w][1] = yB[w]; B[w][2] = zB[w];
  }
  double ssmin = 1E+30, ssc = 0, ttc = 0;
  int ssid = 0;
  for (int ea = 0; ea < 3; ++ea)
    for (int eb = 0; eb < 3; ++eb) {
      double sc, tc;
      const double dist = dor_seg_seg_feature(A[ea], A[(ea + 1) % 3], B[eb], B[(eb + 1) % 3], &sc, &tc);
      if (dist < ssmin) { ssmin = dist; ttc = tc; ssc = sc; ssid = 3 * ea + eb; }
    }
  double ptmin = 1E30, ss = 0, tt = 0;
  int id = 0;
  for (int j = 0; j < 6; ++j) {
    double s, t, dist;
    if (j < 3) dist = dor_pt_tri_feature(A[0], A[1], A[2], B[j], &s, &t);
    else dist = dor_pt_tri_feature(B[0], B[1], B[2], A[j - 3], &s, &t);
    if (dist < ptmin) { ptmin = dist; ss = s; tt = t; id = j; }
  }
  /* the edge-edge switch always writes (zoltan/bf.cpp:497-690) */
  {
    const int ea = ssid / 3, eb = (ssid == 1) ? 2 : ssid % 3; /* case 1 falls into case 2 */
    const double *HA = A[ea], *TA = A[(ea + 1) % 3], *HB = B[eb], *TB = B[(eb + 1) % 3];
    for (int k = 0; k < 3; ++k) {
      pq[k] = TA[k] + ((HA[k] - TA[k]) * ssc);
      pq[3 + k] = TB[k] + ((HB[k] - TB[k]) * ttc);
    }
  }
  if (ptmin > ssmin) return 0; /* zoltan/bf.cpp:891-894 */
  if (id < 3) {
    const int vb = (id == 1) ? 2 : id; /* case 1 falls into case 2 */
    for (int k = 0; k < 3; ++k) {
      pq[k] = A[0][k] + ((A[2][k] - A[0][k]) * tt) + ((A[1][k] - A[0][k]) * ss);
      pq[3 + k] = B[vb][k];
    }
  } else {
    for (int k = 0; k < 3; ++k) {
      pq[k] = A[id - 3][k];
      pq[3 + k] = B[0][k] + ((B[2][k] - B[0][k]) * tt) + ((B[1][k] - B[0][k]) * ss);
    }
  }
  return 0;
}

/* bf(it, nt, A, B, C, D, E, F, P, Q), the SoA shape declared at zoltan/bf.h:61-64 (the
 * reference declares it and defines only the per-pair form): for i in [it, nt), the
 * per-pair bf of triangle (A, B, C) against (D[i], E[i], F[i]); P[i], Q[i] receive its
 * points, and stay untouched where it returns early. */
void dzo_bf_soa(uint32_t it, uint32_t nt, const double a[3], const double b[3], const double c[3], const double *d,
                const double *e, const double *f, int64_t ld, double *p, double *q) {
  const double xA[3] = {a[0], b[0], c[0]}, yA[3] = {a[1], b[1], c[1]}, zA[3] = {a[2], b[2], c[2]};
  for (uint32_t i = it; i < nt; ++i) {
    const double xB[3] = {d[i], e[i], f[i]}, yB[3] = {d[ld + i], e[ld + i], f[ld + i]},
                 zB[3] = {d[2 * ld + i], e[2 * ld + i], f[2 * ld + i]};
    double pq[6];
    if (dzo_bf(xA, yA, zA, xB, yB, zB, pq)) continue;
    for (int k = 0; k < 3; ++k) {
      p[k * ld + i] = pq[k];
      q[k * ld + i] = pq[3 + k];
    }
  }
}

/* The 4x4 quasi-Newton step shared by zoltan/penalty.cpp:95-170 and
 * zoltan/hybrid.cpp:170-249 (the same fused symmetric elimination as penaltySolver,
 * penalty.cpp:395-412 of delta/contact/detection). */
static void zoltan_newton_step(const double A[3], const double D[3], const double BA[3], const double CA[3],
                               const double ED[3], const double FD[3], const double h[16], double r, double delta,
                               const double x[4], double dx[4]) {
  double dh[8], mx[6], a[16], b[4], S[3];
  dh[0] = dh[2] = dh[4] = dh[6] = -1;
  dh[1] = dh[3] = dh[5] = dh[7] = 1;
  if (-x[0] <= 0) dh[0] = mx[0] = 0; else mx[0] = -x[0];
  if (-x[1] <= 0) dh[2] = mx[1] = 0; else mx[1] = -x[1];
  if (x[0] + x[1] - 1 <= 0) dh[1] = dh[3] = mx[2] = 0; else mx[2] = x[0] + x[1] - 1;
  if (-x[2] <= 0) dh[4] = mx[3] = 0; else mx[3] = -x[2];
  if (-x[3] <= 0) dh[6] = mx[4] = 0; else mx[4] = -x[3];
  if (x[2] + x[3] - 1 <= 0) { dh[5] = dh[7] = 0; mx[5] = 0; } else mx[5] = x[2] + x[3] - 1;
  for (int k = 0; k < 3; ++k)
    S[k] = (A[k] + (BA[k] * x[0]) + (CA[k] * x[1])) - (D[k] + (ED[k] * x[2]) + (FD[k] * x[3]));
  b[0] = 2 * dot3z(S, BA) + r * (dh[0] * mx[0] + dh[1] * mx[2]);
  a[0] = h[0] + r * (dh[0] * dh[0] + dh[1] * dh[1]) + delta;
  a[4] = h[4] + r * (dh[3] * dh[1]);
  const double t1 = (h[1] + r * (dh[1] * dh[3])) / a[0];
  a[13] = h[13] - h[12] * t1;
  a[9] = h[9] - h[8] * t1;
  a[5] = (h[5] + r * (dh[2] * dh[2] + dh[3] * dh[3]) + delta) - a[4] * t1;
  b[1] = (2 * dot3z(S, CA) + r * (dh[2] * mx[1] + dh[3] * mx[2])) - b[0] * t1;
  const double t2 = h[2] / a[0];
  const double t3 = h[3] / a[0];
  const double t4 = ((h[6]) - a[4] * t2) / a[5];
  a[14] = ((h[14] + r * (dh[7] * dh[5])) - h[12] * t2) - a[13] * t4;
  a[10] = ((h[10] + r * (dh[4] * dh[4] + dh[5] * dh[5]) + delta) - h[8] * t2) - a[9] * t4;
  b[2] = ((-2 * dot3z(S, ED) + r * (dh[4] * mx[3] + dh[5] * mx[5])) - b[0] * t2) - b[1] * t4;
  const double t5 = (h[7] - a[4] * t3) / a[5];
  const double t6 = (((h[11] + r * (dh[5] * dh[7])) - h[8] * t3) - a[9] * t5) / a[10];
  dx[3] = ((((-2 * dot3z(S, FD) + r * (dh[6] * mx[4] + dh[7] * mx[5])) - b[2] * t6) - b[0] * t3) - b[1] * t5) /
          ((((h[15] + r * (dh[6] * dh[6] + dh[7] * dh[7]) + delta) - h[12] * t3) - a[13] * t5) - a[14] * t6);
  dx[2] = (b[2] - (a[14] * dx[3])) / a[10];
  dx[1] = (b[1] - (a[9] * dx[2] + a[13] * dx[3])) / a[5];
  dx[0] = (b[0] - (a[4] * dx[1] + h[8] * dx[2] + h[12] * dx[3])) / a[0];
}

static void zoltan_hessian(const double BA[3], const double CA[3], const double ED[3], const double FD[3],
                           double h[16]) {
  h[0] = 2. * dot3z(BA, BA);
  h[1] = 2. * dot3z(CA, BA);
  h[2] = -2. * dot3z(ED, BA);
  h[3] = -2. * dot3z(FD, BA);
  h[4] = h[1];
  h[5] = 2. * dot3z(CA, CA);
  h[6] = -2. * dot3z(ED, CA);
  h[7] = -2. * dot3z(FD, CA);
  h[8] = h[2];
  h[9] = h[6];
  h[10] = 2. * dot3z(ED, ED);
  h[11] = 2. * dot3z(FD, ED);
  h[12] = h[3];
  h[13] = h[7];
  h[14] = h[11];
  h[15] = 2. * dot3z(FD, FD);
}

/* ============================================================================
 * zoltan/penalty.cpp:27-209, penalty(it, nt, a, b, c, d, e, f, p, q): for i in [it, nt),
 * 5 quasi-Newton steps from x = 0.33 with delta = 0.1 tr(H), r = lambda 10^(ln lambda
 * + 14) (natural logarithm), and delta multiplied by r before every step when the
 * triangle index i is 4 or more (the test `i < 4` at zoltan/penalty.cpp:137 reads the
 * list index, not the step index).
 * ========================================================================== */
void dzo_penalty_shifted(uint32_t it, uint32_t nt, const double a[3], const double b[3], const double c[3],
                         const double *d, const double *e, const double *f, int64_t ld, double *p, double *q,
                         int32_t r_ulps) {
  for (uint32_t i = it; i < nt; ++i) {
    double A[3], D[3], BA[3], CA[3], ED[3], FD[3], h[16], x[4] = {0.33, 0.33, 0.33, 0.33}, dx[4];
    for (int k = 0; k < 3; ++k) {
      A[k] = a[k];
      D[k] = d[k * ld + i];
      BA[k] = b[k] - a[k];
      CA[k] = c[k] - a[k];
      ED[k] = e[k * ld + i] - d[k * ld + i];
      FD[k] = f[k * ld + i] - d[k * ld + i];
    }
    zoltan_hessian(BA, CA, ED, FD, h);
    const double eps = 0.1;
    double delta = (h[0] + h[5] + h[10] + h[15]) * eps;
    const double lambda = sqrt(0.0125 * (h[0] + h[5] + h[10] + h[15]));
    const double r = shift_ulps_at(lambda * pow(10, log(lambda) + 14), r_ulps, i);
    for (int j = 0; j < 5; ++j) {
      delta = i < 4 ? delta : r * delta;
      zoltan_newton_step(A, D, BA, CA, ED, FD, h, r, delta, x, dx);
      for (int k = 0; k < 4; ++k) x[k] = x[k] - dx[k];
    }
    for (int k = 0; k < 3; ++k) {
      p[k * ld + i] = A[k] + (BA[k] * x[0]) + (CA[k] * x[1]);
      q[k * ld + i] = D[k] + (ED[k] * x[2]) + (FD[k] * x[3]);
    }
  }
}

/* zoltan/hybrid.cpp:134-278: 7 steps with delta = 1e-16 tr(H), r = lambda 10^(log10
 * lambda + 8); error = sqrt(|dx|^2 / |x|^2) of the last step. */
static void zoltan_hybrid_penalty(const double A[3], const double B[3], const double C[3], const double D[3],
                                  const double E[3], const double F[3], double P[3], double Q[3], double *error,
                                  int32_t r_ulps, uint32_t i) {
  double BA[3], CA[3], ED[3], FD[3], h[16], x[4] = {0.33, 0.33, 0.33, 0.33}, dx[4] = {0, 0, 0, 0};
  for (int k = 0; k < 3; ++k) {
    BA[k] = B[k] - A[k];
    CA[k] = C[k] - A[k];
    ED[k] = E[k] - D[k];
    FD[k] = F[k] - D[k];
  }
  zoltan_hessian(BA, CA, ED, FD, h);
  const double eps = 1E-16;
  const double delta = (h[0] + h[5] + h[10] + h[15]) * eps; /* `i < 7 ? delta : 2000*delta` never changes it */
  const double lambda = sqrt(0.0125 * (h[0] + h[5] + h[10] + h[15]));
  const double r = shift_ulps_at(lambda * pow(10, log10(lambda) + 8), r_ulps, i);
  for (int i = 0; i < 7; ++i) {
    zoltan_newton_step(A, D, BA, CA, ED, FD, h, r, delta, x, dx);
    for (int k = 0; k < 4; ++k) x[k] = x[k] - dx[k];
  }
  const double dd = (dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]) + dx[3] * dx[3];
  const double xx = (x[0] * x[0] + x[1] * x[1] + x[2] * x[2]) + x[3] * x[3];
  *error = sqrt(dd / xx);
  for (int k = 0; k < 3; ++k) {
    P[k] = A[k] + (BA[k] * x[0]) + (CA[k] * x[1]);
    Q[k] = D[k] + (ED[k] * x[2]) + (FD[k] * x[3]);
  }
}

/* segt, zoltan/hybrid.cpp:280-342: segment p1p2 against triangle ABC.  Returns 1 when
 * the segment crosses the triangle (P = the crossing), 2 for a segment in the plane, 0
 * or -1 otherwise; P is written whenever the crossing parameter lies in [0, 1], also
 * when the point then falls outside the triangle. */
static int zoltan_segt(const double p1[3], const double p2[3], const double A[3], const double B[3],
                       const double C[3], double P[3]) {
  double u[3], v[3], n[3], dir[3], w0[3], w[3];
  for (int k = 0; k < 3; ++k) {
    u[k] = B[k] - A[k];
    v[k] = C[k] - A[k];
  }
  n[0] = u[1] * v[2] - u[2] * v[1];
  n[1] = u[2] * v[0] - u[0] * v[2];
  n[2] = u[0] * v[1] - u[1] * v[0];
  if (n[0] == 0 && n[1] == 0 && n[2] == 0) return -1;
  for (int k = 0; k < 3; ++k) {
    dir[k] = p2[k] - p1[k];
    w0[k] = p1[k] - A[k];
  }
  const double a = -dot3z(n, w0);
  const double b = dot3z(n, dir);
  if (fabs(b) < 1E-99 && a == 0) return 2;
  const double r = a / b;
  if (r < 0.0 || r > 1.0) return 0; /* `r == NAN` (hybrid.cpp:309) is always false */
  for (int k = 0; k < 3; ++k) P[k] = p1[k] + r * dir[k];
  const double uu = dot3z(u, u), uv = dot3z(u, v), vv = dot3z(v, v);
  for (int k = 0; k < 3; ++k) w[k] = P[k] - A[k];
  const double wu = dot3z(w, u), wv = dot3z(w, v);
  const double D = uv * uv - uu * vv;
  const double s = (uv * wv - vv * wu) / D;
  if (s < 0.0 || s > 1.0) return 0;
  const double t = (uv * wu - uu * wv) / D;
  if (t < 0.0 || (s + t) > 1.0) return 0;
  return 1;
}

/* segseg, zoltan/hybrid.cpp:344-445: Sunday's parameters with SMALL_NUM = 1e-8.  Q's y
 * and z start from p4's x (Q[1] = p4[0] + ..., Q[2] = p4[0] + ..., hybrid.cpp:436-437);
 * the returned distance is that of the correct points. */
static double zoltan_segseg(const double p1[3], const double p2[3], const double p3[3], const double p4[3],
                            double P[3], double Q[3]) {
  double u[3], v[3], w[3];
  for (int k = 0; k < 3; ++k) {
    u[k] = p1[k] - p2[k];
    v[k] = p3[k] - p4[k];
    w[k] = p2[k] - p4[k];
  }
  const double a = dot3z(u, u), b = dot3z(u, v), c = dot3z(v, v), d = dot3z(u, w), e = dot3z(v, w);
  const double D = a * c - b * b;
  double sD = D, tD = D, sN = 0, tN = 0;
  const double SMALL_NUM = 0.00000001;
  if (D < SMALL_NUM) {
    sN = 0.0; sD = 1.0; tN = e; tD = c;
  } else {
    sN = (b * e - c * d);
    tN = (a * e - b * d);
    if (sN < 0.0) { sN = 0.0; tN = e; tD = c; }
    else if (sN > sD) { sN = sD; tN = e + b; tD = c; }
  }
  if (tN < 0.0) {
    tN = 0.0;
    if (-d < 0.0) sN = 0.0;
    else if (-d > a) sN = sD;
    else { sN = -d; sD = a; }
  } else if (tN > tD) {
    tN = tD;
    if ((-d + b) < 0.0) sN = 0;
    else if ((-d + b) > a) sN = sD;
    else { sN = (-d + b); sD = a; }
  }
  const double sc = (fabs(sN) < SMALL_NUM) ? 0.0 : sN / sD;
  const double tc = (fabs(tN) < SMALL_NUM) ? 0.0 : tN / tD;
  for (int k = 0; k < 3; ++k) P[k] = p2[k] + u[k] * sc;
  Q[0] = p4[0] + v[0] * tc;
  Q[1] = p4[0] + v[1] * tc;
  Q[2] = p4[0] + v[2] * tc;
  double dP[3];
  for (int k = 0; k < 3; ++k) dP[k] = w[k] + (sc * u[k]) - (tc * v[k]);
  return sqrt(dot3z(dP, dP));
}

/* bf, zoltan/hybrid.cpp:646-886: the six segment-triangle crossings first (a crossing
 * gives Q = P = the crossing point), else the minimum over 6 vertex-face and 9 edge-edge
 * features; on a tie the edge-edge point on A and the vertex-face point on B.  P and Q
 * are in/out: with NaN distances no branch writes them. */
static void zoltan_hybrid_bf(const double A[3], const double B[3], const double C[3], const double D[3],
                             const double E[3], const double F[3], double P[3], double Q[3]) {
  int intersection = 0;
  if (zoltan_segt(D, E, A, B, C, P) == 1) intersection = 1;
  else if (zoltan_segt(E, F, A, B, C, P) == 1) intersection = 1;
  else if (zoltan_segt(F, D, A, B, C, P) == 1) intersection = 1;
  else if (zoltan_segt(A, B, D, E, F, P) == 1) intersection = 1;
  else if (zoltan_segt(B, C, D, E, F, P) == 1) intersection = 1;
  else if (zoltan_segt(C, A, D, E, F, P) == 1) intersection = 1;
  double tp[3] = {0, 0, 0}, tq[3] = {0, 0, 0}, tmpP[3], tmpQ[3], ssP[3] = {0, 0, 0}, ssQ[3] = {0, 0, 0};
  double ptmin = 1E+30, ssmin = 1E+30, tmp;
  if (intersection != 1) {
    const double *av[3] = {A, B, C}, *bv[3] = {D, E, F};
    for (int j = 0; j < 3; ++j) { /* vertices of A against triangle DEF */
      tmp = dor_pt(D, E, F, av[j], tmpP);
      if (j == 0 || ptmin > tmp) {
        ptmin = tmp;
        memcpy(tp, av[j], sizeof tp);
        memcpy(tq, tmpP, sizeof tq);
      }
    }
    for (int j = 0; j < 3; ++j) { /* vertices of B against triangle ABC */
      tmp = dor_pt(A, B, C, bv[j], tmpP);
      if (ptmin > tmp) {
        ptmin = tmp;
        memcpy(tq, bv[j], sizeof tq);
        memcpy(tp, tmpP, sizeof tp);
      }
    }
    for (int ea = 0; ea < 3; ++ea)
      for (int eb = 0; eb < 3; ++eb) {
        tmp = zoltan_segseg(av[ea], av[(ea + 1) % 3], bv[eb], bv[(eb + 1) % 3], tmpP, tmpQ);
        if ((ea == 0 && eb == 0) || ssmin > tmp) {
          ssmin = tmp;
          memcpy(ssP, tmpP, sizeof ssP);
          memcpy(ssQ, tmpQ, sizeof ssQ);
        }
      }
  }
  if (intersection == 1) {
    memcpy(Q, P, 3 * sizeof(double));
  } else if (ssmin < ptmin) {
    memcpy(P, ssP, 3 * sizeof(double));
    memcpy(Q, ssQ, 3 * sizeof(double));
  } else if (ssmin > ptmin) {
    memcpy(P, tp, 3 * sizeof(double));
    memcpy(Q, tq, 3 * sizeof(double));
  } else if (ssmin == ptmin) {
    memcpy(P, ssP, 3 * sizeof(double));
    memcpy(Q, tq, 3 * sizeof(double));
  }
}

/* ============================================================================
 * zoltan/hybrid.cpp:37-131, hybrid(it, nt, a, b, c, d, e, f, p, q), in its serial
 * meaning: batches k in [it, nt/4) of the 4 triangles 4k..4k+3 (`it` counts batches;
 * the triangles past the last full batch are not visited).  Each triangle gets the
 * 7-step penalty points; when the batch's mean error exceeds 1e-8, every triangle of the
 * batch gets the points of bf with the batch's last triangle (the loop at
 * hybrid.cpp:115-128 reuses the A..F left by the penalty loop).
 * ========================================================================== */
void dzo_hybrid_shifted(int32_t it, int32_t nt, const double a[3], const double b[3], const double c[3],
                        const double *d, const double *e, const double *f, int64_t ld, double *p, double *q,
                        int32_t r_ulps, int32_t mode) {
  const unsigned batchSize = 4;
  double D[3] = {0, 0, 0}, E[3] = {0, 0, 0}, F[3] = {0, 0, 0}, P[3] = {0, 0, 0}, Q[3] = {0, 0, 0};
  for (unsigned k = (unsigned)it; k < (unsigned)nt / batchSize; k++) {
    double error[4];
    for (unsigned l = 0; l < batchSize; l++) {
      const unsigned i = k * batchSize + l;
      for (int x = 0; x < 3; ++x) {
        D[x] = d[x * ld + i];
        E[x] = e[x * ld + i];
        F[x] = f[x * ld + i];
      }
      zoltan_hybrid_penalty(a, b, c, D, E, F, P, Q, &error[l], r_ulps, i);
      for (int x = 0; x < 3; ++x) {
        p[x * ld + i] = P[x];
        q[x * ld + i] = Q[x];
      }
    }
    double batchError = 0.0;
    for (unsigned l = 0; l < batchSize; l++) batchError += error[l];
    /* mode 0: the reference's decision; 1: never fall back; 2: always fall back */
    if (mode == 2 || (mode == 0 && batchError / batchSize > 1E-8)) {
      for (unsigned l = 0; l < batchSize; l++) {
        const unsigned i = k * batchSize + l;
        zoltan_hybrid_bf(a, b, c, D, E, F, P, Q);
        for (int x = 0; x < 3; ++x) {
          p[x * ld + i] = P[x];
          q[x * ld + i] = Q[x];
        }
      }
    }
  }
}

/* ============================================================================
 * zoltan/dynamics.cpp
 * ========================================================================== */
/* TVMUL, NVMUL, NNMUL, NVADDMUL of zoltan/algo.h: matrices column-major (A[3*col+row]). */
static void tvmul(const double *A, const double *B, double *C) {
  C[0] = A[0] * B[0] + A[1] * B[1] + A[2] * B[2];
  C[1] = A[3] * B[0] + A[4] * B[1] + A[5] * B[2];
  C[2] = A[6] * B[0] + A[7] * B[1] + A[8] * B[2];
}
static void nvmul(const double *A, const double *B, double *C) {
  C[0] = A[0] * B[0] + A[3] * B[1] + A[6] * B[2];
  C[1] = A[1] * B[0] + A[4] * B[1] + A[7] * B[2];
  C[2] = A[2] * B[0] + A[5] * B[1] + A[8] * B[2];
}
static void nnmul(const double *A, const double *B, double *C) {
  for (int col = 0; col < 3; ++col)
    for (int row = 0; row < 3; ++row)
      C[3 * col + row] = A[row] * B[3 * col] + A[3 + row] * B[3 * col + 1] + A[6 + row] * B[3 * col + 2];
}
static void nvaddmul(const double *C, const double *A, const double *B, double *D) {
  const double d0 = C[0] + (A[0] * B[0] + A[3] * B[1] + A[6] * B[2]);
  const double d1 = C[1] + (A[1] * B[0] + A[4] * B[1] + A[7] * B[2]);
  const double d2 = C[2] + (A[2] * B[0] + A[5] * B[1] + A[8] * B[2]);
  D[0] = d0; D[1] = d1; D[2] = d2;
}

/* dynamics::update, zoltan/dynamics.cpp:66-250.  Per body: read force and torque and
 * zero them; half-step angular momentum with expmap(-h/2 O), gyroscopic term, O(t+h);
 * v += (step/m) f; rotation L2 = L1 expmap(step O); spatial angular velocity o = L2 O;
 * x += step v.  Then every triangle's three spatial vertices from its referential ones:
 * x + L (X_ref - X_centre).  expmap is dynamics.cpp:338-414, the same function as
 * delta/dynamics/dynamics.cpp:26-102 (its v02 = Omega2*Omega3 included). */
void dzo_update(int32_t nt, int32_t nb, double *t, int64_t ldt, const int32_t *pid, double *angular,
                double *linear, double *rotation, double *position, const double *inertia, const double *inverse,
                const double *mass, double *force, double *torque, double step) {
  const double half = 0.5 * step;
  for (int i = 0; i < nb; i++) {
    double O[3], v[3], L1[9], J[9], I[9], im, f[3], tq[3], T[3], DL[9], L2[9], A[3], B[3], o[3];
    for (int k = 0; k < 3; ++k) {
      O[k] = angular[k * nb + i];
      v[k] = linear[k * nb + i];
      f[k] = force[k * nb + i];
      tq[k] = torque[k * nb + i];
      force[k * nb + i] = 0.0;
      torque[k * nb + i] = 0.0;
    }
    for (int k = 0; k < 9; ++k) {
      L1[k] = rotation[k * nb + i];
      J[k] = inertia[k * nb + i];
      I[k] = inverse[k * nb + i];
    }
    im = 1 / mass[i];
    tvmul(L1, tq, T);
    dor_expmap(-half * O[0], -half * O[1], -half * O[2], DL);
    nvmul(J, O, A);
    nvmul(DL, A, B);
    for (int k = 0; k < 3; ++k) B[k] = B[k] + (half) * T[k]; /* ADDMUL(B, half, T, B) */
    nvmul(I, B, A);
    nvmul(J, A, B);
    T[0] -= A[1] * B[2] - A[2] * B[1]; /* PRODUCTSUB(A, B, T) */
    T[1] -= A[2] * B[0] - A[0] * B[2];
    T[2] -= A[0] * B[1] - A[1] * B[0];
    for (int k = 0; k < 3; ++k) T[k] *= step;
    nvaddmul(O, I, T, O);
    im *= step;
    for (int k = 0; k < 3; ++k) v[k] = v[k] + (im) * f[k]; /* ADDMUL(v, im, f, v) */
    dor_expmap(step * O[0], step * O[1], step * O[2], DL);
    nnmul(L1, DL, L2);
    for (int k = 0; k < 9; ++k) rotation[k * nb + i] = L2[k];
    nvmul(L2, O, o);
    for (int k = 0; k < 3; ++k) {
      position[k * nb + i] += step * v[k];
      angular[k * nb + i] = O[k];
      angular[(3 + k) * nb + i] = o[k];
      linear[k * nb + i] = v[k];
    }
  }
  for (int i = 0; i < nt; i++) {
    const int j = pid[i];
    double L[9], X[3], x[3], C[3], c[3];
    for (int k = 0; k < 9; ++k) L[k] = rotation[k * nb + j];
    for (int k = 0; k < 3; ++k) {
      X[k] = position[(3 + k) * nb + j];
      x[k] = position[k * nb + j];
    }
    for (int w = 0; w < 3; ++w) {
      for (int k = 0; k < 3; ++k) C[k] = t[(3 * (3 + w) + k) * ldt + i] - X[k]; /* SCC(X, C) */
      nvaddmul(x, L, C, c);
      for (int k = 0; k < 3; ++k) t[(3 * w + k) * ldt + i] = c[k];
    }
  }
}

/* dynamics::euler, zoltan/dynamics.cpp:252-297 */
void dzo_euler(int32_t nb, double *angular, const double *linear, double *rotation, double *position, double step) {
  for (int i = 0; i < nb; i++) {
    double O[3], L1[9], DL[9], L2[9], o[3];
    for (int k = 0; k < 3; ++k) O[k] = angular[k * nb + i];
    dor_expmap(step * O[0], step * O[1], step * O[2], DL);
    for (int k = 0; k < 9; ++k) L1[k] = rotation[k * nb + i];
    nnmul(L1, DL, L2);
    for (int k = 0; k < 9; ++k) rotation[k * nb + i] = L2[k];
    nvmul(L2, O, o);
    for (int k = 0; k < 3; ++k) angular[(3 + k) * nb + i] = o[k];
    for (int k = 0; k < 3; ++k) position[k * nb + i] += step * linear[k * nb + i];
  }
}

/* dynamics::integrate, zoltan/dynamics.cpp:299-335: each triangle's three vertices move
 * by step v; a velocity component flips sign for every vertex coordinate outside
 * [lo, hi] (checked vertex by vertex, so it can flip more than once). */
void dzo_integrate(double step, const double lo[3], const double hi[3], int32_t nt, double *t, int64_t ldt,
                   double *v) {
  for (int i = 0; i < nt; i++) {
    for (int w = 0; w < 3; ++w)
      for (int k = 0; k < 3; ++k) t[(3 * w + k) * ldt + i] += step * v[k * ldt + i];
    for (int w = 0; w < 3; ++w) {
      for (int k = 0; k < 3; ++k)
        if (t[(3 * w + k) * ldt + i] < lo[k]) v[k * ldt + i] *= -1;
      for (int k = 0; k < 3; ++k)
        if (t[(3 * w + k) * ldt + i] > hi[k]) v[k * ldt + i] *= -1;
    }
  }
}

/* ============================================================================
 * forces::force, zoltan/forces.cpp:48-205, on one process (loba_query answers this
 * rank, the force migration has nothing to send).  Contacts are grouped by master body:
 * body i's contacts are [offset[i], offset[i+1]) with slave[], point[], normal[], depth[]
 * (the normal and depth as the caller's contactpoint holds them).  For i = 0..nb-1 in
 * order, each contact k of i adds granular's f = (kn depth + en vn) n (forces.cpp:28-44;
 * en = damper sqrt(kn m_red)) to i's force and (p - x_i) x f to its torque, and -f and
 * (p - x_j) x (-f) to the slave j; then i's force gets mass_i gravity.  force and torque
 * accumulate onto their inputs.
 * ========================================================================== */
void dzo_force(int32_t nb, const int64_t *offset, const int32_t *slave, const double *point, const double *normal,
               const double *depth, int64_t ldc, const double *position, const double *angular, const double *linear,
               const double *mass, double *force, double *torque, const double gravity[3], double spring,
               double damper) {
  for (int i = 0; i < nb; i++) {
    double oi[3], v[3], x[3];
    for (int k = 0; k < 3; ++k) {
      oi[k] = angular[(3 + k) * nb + i];
      v[k] = linear[k * nb + i];
      x[k] = position[k * nb + i];
    }
    for (int64_t c = offset[i]; c < offset[i + 1]; ++c) {
      double p[3], z[3], vi[3], vj[3], oj[3], vij[3], n[3], a[3], f[3];
      for (int k = 0; k < 3; ++k) {
        p[k] = point[k * ldc + c];
        n[k] = normal[k * ldc + c];
      }
      for (int k = 0; k < 3; ++k) z[k] = p[k] - x[k];
      vi[0] = oi[1] * z[2] - oi[2] * z[1] + v[0];
      vi[1] = oi[2] * z[0] - oi[0] * z[2] + v[1];
      vi[2] = oi[0] * z[1] - oi[1] * z[0] + v[2];
      const int j = slave[c];
      for (int k = 0; k < 3; ++k) {
        z[k] = p[k] - position[k * nb + j];
        oj[k] = angular[(3 + k) * nb + j];
      }
      vj[0] = oj[1] * z[2] - oj[2] * z[1] + linear[0 * nb + j];
      vj[1] = oj[2] * z[0] - oj[0] * z[2] + linear[1 * nb + j];
      vj[2] = oj[0] * z[1] - oj[1] * z[0] + linear[2 * nb + j];
      for (int k = 0; k < 3; ++k) vij[k] = vj[k] - vi[k];
      /* granular, forces.cpp:28-44 */
      const double ma = 1.0 / ((1 / mass[i]) + (1 / mass[j]));
      const double kn = spring;
      const double en = damper * sqrt(kn * ma);
      const double vn = dot3z(vij, n);
      const double fn = (kn * depth[c]) + (en * vn);
      for (int k = 0; k < 3; ++k) f[k] = fn * n[k];
      for (int k = 0; k < 3; ++k) force[k * nb + i] += f[k];
      for (int k = 0; k < 3; ++k) a[k] = p[k] - x[k];
      torque[0 * nb + i] += a[1] * f[2] - a[2] * f[1];
      torque[1 * nb + i] += a[2] * f[0] - a[0] * f[2];
      torque[2 * nb + i] += a[0] * f[1] - a[1] * f[0];
      for (int k = 0; k < 3; ++k) f[k] = -f[k];
      for (int k = 0; k < 3; ++k) force[k * nb + j] += f[k];
      for (int k = 0; k < 3; ++k) a[k] = p[k] - position[k * nb + j];
      torque[0 * nb + j] += a[1] * f[2] - a[2] * f[1];
      torque[1 * nb + j] += a[2] * f[0] - a[0] * f[2];
      torque[2 * nb + j] += a[0] * f[1] - a[1] * f[0];
    }
    for (int k = 0; k < 3; ++k) force[k * nb + i] += mass[i] * gravity[k];
  }
}

void dzo_penalty(uint32_t it, uint32_t nt, const double a[3], const double b[3], const double c[3],
                 const double *d, const double *e, const double *f, int64_t ld, double *p, double *q) {
  dzo_penalty_shifted(it, nt, a, b, c, d, e, f, ld, p, q, 0);
}

void dzo_hybrid(int32_t it, int32_t nt, const double a[3], const double b[3], const double c[3], const double *d,
                const double *e, const double *f, int64_t ld, double *p, double *q) {
  dzo_hybrid_shifted(it, nt, a, b, c, d, e, f, ld, p, q, 0, 0);
}
