/*
 * delta_oracle.c -- CPU restatement (FP64) of the reference's contact hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker).  See delta_oracle.h for the layouts.
 * Compile with -ffp-contract=off: the floating-point operation order below is the
 * reference's, term by term, so that results are bit-identical to the reference
 * compiled without FMA contraction.  Reference paths are relative to the project root.
 */
#include "delta_oracle.h"
#include "oracle_internal.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

static inline double dot3(const double *a, const double *b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

/* ============================================================================
 * bfSolver, bf.cpp:217-1178
 *
 * Minimum over 9 edge-edge features (bf.cpp:586-713) and 6 vertex-face features
 * (bf.cpp:920-1100).  Edge e of a triangle V runs from its tail V[(e+1)%3]
 * (parameter 0) to its head V[e] (parameter 1); edge pair j = 3*eA + eB.  The
 * segment-triangle loop at bf.cpp:359-407 reads uninitialised data and its
 * result is always overwritten, so it has no effect and is not restated.
 * ========================================================================== */

/* One edge-edge feature: clamped closest parameters (Sunday's method as written
 * in bf.cpp:586-697) and the distance of the resulting point pair. */
double dor_seg_seg_feature(const double *HA, const double *TA, const double *HB,
                              const double *TB, double *sc_out, double *tc_out) {
  double u[3], v[3], w[3];
  for (int k = 0; k < 3; ++k) {
    u[k] = HA[k] - TA[k];
    v[k] = HB[k] - TB[k];
    w[k] = TA[k] - TB[k];
  }
  const double a = dot3(u, u), b = dot3(u, v), c = dot3(v, v);
  const double d = dot3(u, w), e = dot3(v, w);
  const double D = a * c - b * b;
  const double SMALL = 1e-30;
  double sD = D, tD = D, sN, tN;
  if (D < SMALL) {
    sN = 0.0;
    sD = 1.0;
    tN = e;
    tD = c;
  } else {
    sN = b * e - c * d;
    tN = a * e - b * d;
    if (sN < 0.0) {
      sN = 0.0;
      tN = e;
      tD = c;
    } else if (sN > sD) {
      sN = sD;
      tN = e + b;
      tD = c;
    }
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
  const double sc = (fabs(sN) < SMALL) ? 0.0 : sN / sD;
  const double tc = (fabs(tN) < SMALL) ? 0.0 : tN / tD;
  double dP[3];
  for (int k = 0; k < 3; ++k) dP[k] = (TA[k] - TB[k]) + (sc * (HA[k] - TA[k])) - (tc * (HB[k] - TB[k]));
  *sc_out = sc;
  *tc_out = tc;
  return sqrt(dP[0] * dP[0] + dP[1] * dP[1] + dP[2] * dP[2]);
}

/* One vertex-face feature: point X against triangle (V0,V1,V2), Eberly's region
 * classification as written in bf.cpp:920-1090.  Returns the distance, and the
 * parameters s (along V1-V0) and t (along V2-V0). */
double dor_pt_tri_feature(const double *V0, const double *V1, const double *V2,
                             const double *X, double *s_out, double *t_out) {
  double E0[3], E1[3], Dv[3];
  for (int k = 0; k < 3; ++k) {
    E0[k] = V1[k] - V0[k];
    E1[k] = V2[k] - V0[k];
    Dv[k] = V0[k] - X[k];
  }
  const double a = dot3(E0, E0), b = dot3(E0, E1), c = dot3(E1, E1);
  const double d = dot3(E0, Dv), e = dot3(E1, Dv), f = dot3(Dv, Dv);
  const double det = a * c - b * b;
  double s = b * e - c * d;
  double t = b * d - a * e;
  double sq = 0.0;
#define FULLQ (s * (a * s + b * t + 2 * d) + t * (b * s + c * t + 2 * e) + f)
  if ((s + t) <= det) {
    if (s < 0) {
      if (t < 0) { /* region 4 */
        if (d < 0) {
          t = 0;
          if (-d >= a) { s = 1; sq = a + 2 * d + f; }
          else { s = -d / a; sq = d * s + f; }
        } else {
          s = 0;
          if (e >= 0) { t = 0; sq = f; }
          else if (-e >= c) { t = 1; sq = c + 2 * e + f; }
          else { t = -e / c; sq = e * t + f; }
        }
      } else { /* region 3 */
        s = 0;
        if (e >= 0) { t = 0; sq = f; }
        else if (-e >= c) { t = 1; sq = c + 2 * e + f; }
        else { t = -e / c; sq = e * t + f; }
      }
    } else if (t < 0) { /* region 5 */
      t = 0;
      if (d >= 0) { s = 0; sq = f; }
      else if (-d >= a) { s = 1; sq = a + 2 * d + f; }
      else { s = -d / a; sq = d * s + f; }
    } else { /* region 0 */
      const double inv = 1 / det;
      s = s * inv;
      t = t * inv;
      sq = FULLQ;
    }
  } else {
    if (s < 0) { /* region 2 */
      const double tmp0 = b + d, tmp1 = c + e;
      if (tmp1 > tmp0) {
        const double numer = tmp1 - tmp0, denom = a - 2 * b + c;
        if (numer >= denom) { s = 1; t = 0; sq = a + 2 * d + f; }
        else { s = numer / denom; t = 1 - s; sq = FULLQ; }
      } else {
        s = 0;
        if (tmp1 <= 0) { t = 1; sq = c + 2 * e + f; }
        else if (e >= 0) { t = 0; sq = f; }
        else { t = -e / c; sq = e * t + f; }
      }
    } else if (t < 0) { /* region 6 */
      const double tmp0 = b + e, tmp1 = a + d;
      if (tmp1 > tmp0) {
        const double numer = tmp1 - tmp0, denom = a - 2 * b + c;
        if (numer >= denom) { t = 1; s = 0; sq = c + 2 * e + f; }
        else { t = numer / denom; s = 1 - t; sq = FULLQ; }
      } else {
        t = 0;
        if (tmp1 <= 0) { s = 1; sq = a + 2 * d + f; }
        else if (d >= 0) { s = 0; sq = f; }
        else { s = -d / a; sq = d * s + f; }
      }
    } else { /* region 1 */
      const double numer = c + e - b - d;
      if (numer <= 0) { s = 0; t = 1; sq = c + 2 * e + f; }
      else {
        const double denom = a - 2 * b + c;
        if (numer >= denom) { s = 1; t = 0; sq = a + 2 * d + f; }
        else { s = numer / denom; t = 1 - s; sq = FULLQ; }
      }
    }
  }
#undef FULLQ
  if (sq <= 0.0) sq = 0.0;
  *s_out = s;
  *t_out = t;
  return sqrt(sq);
}

void dor_bf_solver(const double *xA, const double *yA, const double *zA,
                   const double *xB, const double *yB, const double *zB, double pq[6]) {
  double A[3][3], B[3][3];
  for (int v = 0; v < 3; ++v) {
    A[v][0] = xA[v]; A[v][1] = yA[v]; A[v][2] = zA[v];
    B[v][0] = xB[v]; B[v][1] = yB[v]; B[v][2] = zB[v];
  }
  /* edge-edge minimum, first minimum wins (bf.cpp:698-705) */
  double ssmin = 1E+30, ssc = 0, ttc = 0;
  int ssid = 0;
  for (int ea = 0; ea < 3; ++ea)
    for (int eb = 0; eb < 3; ++eb) {
      double sc, tc;
      const double dist = dor_seg_seg_feature(A[ea], A[(ea + 1) % 3], B[eb], B[(eb + 1) % 3], &sc, &tc);
      if (dist < ssmin) { ssmin = dist; ttc = tc; ssc = sc; ssid = 3 * ea + eb; }
    }
  /* vertex-face minimum: B's vertices against A (j=0..2), A's against B (j=3..5) */
  double ptmin = 1E30, ss = 0.0, tt = 0.0;
  int id = 0;
  for (int j = 0; j < 6; ++j) {
    double s, t, dist;
    if (j < 3) dist = dor_pt_tri_feature(A[0], A[1], A[2], B[j], &s, &t);
    else dist = dor_pt_tri_feature(B[0], B[1], B[2], A[j - 3], &s, &t);
    if (dist < ptmin) { ptmin = dist; ss = s; tt = t; id = j; }
  }
  if (ptmin > ssmin) { /* bf.cpp:1102 */
    const int ea = ssid / 3, eb = ssid % 3;
    const double *HA = A[ea], *TA = A[(ea + 1) % 3], *HB = B[eb], *TB = B[(eb + 1) % 3];
    for (int k = 0; k < 3; ++k) {
      pq[k] = TA[k] + ((HA[k] - TA[k]) * ssc);
      pq[3 + k] = TB[k] + ((HB[k] - TB[k]) * ttc);
    }
    return;
  }
  if (id < 3) {
    for (int k = 0; k < 3; ++k) {
      pq[k] = A[0][k] + ((A[2][k] - A[0][k]) * tt) + ((A[1][k] - A[0][k]) * ss);
      pq[3 + k] = B[id][k];
    }
  } else {
    for (int k = 0; k < 3; ++k) {
      pq[k] = A[id - 3][k];
      pq[3 + k] = B[0][k] + ((B[2][k] - B[0][k]) * tt) + ((B[1][k] - B[0][k]) * ss);
    }
  }
}

/* ============================================================================
 * penaltySolver, penalty.cpp:278-432 (fixed 4 iterations, `failed`) and
 * penalty.cpp:434-582 (at most 16 iterations, early exit).  Unknowns x[0..3] are the
 * barycentric weights of BA, CA (triangle A) and ED, FD (triangle B).
 * ========================================================================== */
static void penalty_common(const double *xA, const double *yA, const double *zA,
                           const double *xB, const double *yB, const double *zB,
                           double max_error, int adaptive, double pq[6],
                           int32_t *failed, int32_t *iterations) {
  double A0[3] = {xA[0], yA[0], zA[0]}, B0[3] = {xB[0], yB[0], zB[0]};
  double BA[3] = {xA[1] - xA[0], yA[1] - yA[0], zA[1] - zA[0]};
  double CA[3] = {xA[2] - xA[0], yA[2] - yA[0], zA[2] - zA[0]};
  double ED[3] = {xB[1] - xB[0], yB[1] - yB[0], zB[1] - zB[0]};
  double FD[3] = {xB[2] - xB[0], yB[2] - yB[0], zB[2] - zB[0]};
  double h[16];
  h[0] = 2. * dot3(BA, BA);
  h[1] = 2. * dot3(CA, BA);
  h[2] = -2. * dot3(ED, BA);
  h[3] = -2. * dot3(FD, BA);
  h[4] = h[1];
  h[5] = 2. * dot3(CA, CA);
  h[6] = -2. * dot3(ED, CA);
  h[7] = -2. * dot3(FD, CA);
  h[8] = h[2];
  h[9] = h[6];
  h[10] = 2. * dot3(ED, ED);
  h[11] = 2. * dot3(FD, ED);
  h[12] = h[3];
  h[13] = h[7];
  h[14] = h[11];
  h[15] = 2. * dot3(FD, FD);
  const double eps = 1E-2;
  double delta = (h[0] + h[5] + h[10] + h[15]) * eps;
  const double lambda = sqrt(0.0125 * (h[0] + h[5] + h[10] + h[15]));
  const double r = lambda * 1E5;
  double x[4] = {0.33, 0.33, 0.33, 0.33};
  const int n_iter = adaptive ? 16 : 4; /* MaxNumberOfNewtonIterations, penalty.h:38 */
  if (failed) *failed = 0;
  for (int i = 0; i < n_iter; ++i) {
    double dh[8], mx[6], dx[4], a[16], b[4], S[3];
    /* active-constraint gradients and violations (penalty.cpp:367-383) */
    dh[0] = (-x[0] <= 0) ? 0.0 : -1;
    mx[0] = (-x[0] <= 0) ? 0.0 : -x[0];
    dh[2] = (-x[1] <= 0) ? 0.0 : -1;
    mx[1] = (-x[1] <= 0) ? 0.0 : -x[1];
    dh[1] = dh[3] = (x[0] + x[1] - 1 <= 0) ? 0.0 : 1;
    mx[2] = (x[0] + x[1] - 1 <= 0) ? 0.0 : x[0] + x[1] - 1;
    dh[4] = (-x[2] <= 0) ? 0.0 : -1;
    mx[3] = (-x[2] <= 0) ? 0.0 : -x[2];
    dh[6] = (-x[3] <= 0) ? 0.0 : -1;
    mx[4] = (-x[3] <= 0) ? 0.0 : -x[3];
    dh[5] = dh[7] = (x[2] + x[3] - 1 <= 0) ? 0.0 : 1;
    mx[5] = (x[2] + x[3] - 1 <= 0) ? 0.0 : x[2] + x[3] - 1;
    if (adaptive) delta = i < 3 ? delta : 1E5 * delta; /* penalty.cpp:533 */
    for (int k = 0; k < 3; ++k)
      S[k] = (A0[k] + (BA[k] * x[0]) + (CA[k] * x[1])) - (B0[k] + (ED[k] * x[2]) + (FD[k] * x[3]));
    /* fused symmetric elimination of the 4x4 system (penalty.cpp:395-412) */
    b[0] = 2 * dot3(S, BA) + r * (dh[0] * mx[0] + dh[1] * mx[2]);
    a[0] = h[0] + r * (dh[0] * dh[0] + dh[1] * dh[1]) + delta;
    a[4] = h[4] + r * (dh[3] * dh[1]);
    const double t1 = (h[1] + r * (dh[1] * dh[3])) / a[0];
    a[13] = h[13] - h[12] * t1;
    a[9] = h[9] - h[8] * t1;
    a[5] = (h[5] + r * (dh[2] * dh[2] + dh[3] * dh[3]) + delta) - a[4] * t1;
    b[1] = (2 * dot3(S, CA) + r * (dh[2] * mx[1] + dh[3] * mx[2])) - b[0] * t1;
    const double t2 = h[2] / a[0];
    const double t3 = h[3] / a[0];
    const double t4 = ((h[6]) - a[4] * t2) / a[5];
    a[14] = ((h[14] + r * (dh[7] * dh[5])) - h[12] * t2) - a[13] * t4;
    a[10] = ((h[10] + r * (dh[4] * dh[4] + dh[5] * dh[5]) + delta) - h[8] * t2) - a[9] * t4;
    b[2] = ((-2 * dot3(S, ED) + r * (dh[4] * mx[3] + dh[5] * mx[5])) - b[0] * t2) - b[1] * t4;
    const double t5 = (h[7] - a[4] * t3) / a[5];
    const double t6 = (((h[11] + r * (dh[5] * dh[7])) - h[8] * t3) - a[9] * t5) / a[10];
    dx[3] = ((((-2 * dot3(S, FD) + r * (dh[6] * mx[4] + dh[7] * mx[5])) - b[2] * t6) - b[0] * t3) - b[1] * t5) /
            ((((h[15] + r * (dh[6] * dh[6] + dh[7] * dh[7]) + delta) - h[12] * t3) - a[13] * t5) - a[14] * t6);
    dx[2] = (b[2] - (a[14] * dx[3])) / a[10];
    dx[1] = (b[1] - (a[9] * dx[2] + a[13] * dx[3])) / a[5];
    dx[0] = (b[0] - (a[4] * dx[1] + h[8] * dx[2] + h[12] * dx[3])) / a[0];
    const double dxx = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2] + dx[3] * dx[3];
    const double xx = x[0] * x[0] + x[1] * x[1] + x[2] * x[2] + x[3] * x[3];
    if (adaptive) {
      const double error = dxx / xx;
      if (error < max_error * max_error) {
        if (iterations) *iterations = i;
        break;
      }
    } else {
      delta = 1E4 * delta;
      if (failed) *failed = (dxx / xx > max_error * max_error) ? 1 : 0;
    }
    x[0] = x[0] - dx[0];
    x[1] = x[1] - dx[1];
    x[2] = x[2] - dx[2];
    x[3] = x[3] - dx[3];
  }
  for (int k = 0; k < 3; ++k) {
    pq[k] = A0[k] + (BA[k] * x[0]) + (CA[k] * x[1]);
    pq[3 + k] = B0[k] + (ED[k] * x[2]) + (FD[k] * x[3]);
  }
}

void dor_penalty_solver(const double *xA, const double *yA, const double *zA,
                        const double *xB, const double *yB, const double *zB,
                        double max_error, double pq[6], int32_t *failed) {
  penalty_common(xA, yA, zA, xB, yB, zB, max_error, 0, pq, failed, NULL);
}

/* The iteration count is written only on early exit, as in penalty.cpp:559-562;
 * the caller's initial value survives otherwise. */
void dor_penalty_solver_iter(const double *xA, const double *yA, const double *zA,
                             const double *xB, const double *yB, const double *zB,
                             double max_error, double pq[6], int32_t *iterations) {
  penalty_common(xA, yA, zA, xB, yB, zB, max_error, 1, pq, NULL, iterations);
}

/* ============================================================================
 * GJK with Johnson's sub-simplex projection, gjk.cpp:102-460 (Solfec).
 * ========================================================================== */
typedef struct { double w[3]; const double *a, *b; } gjk_point;

/* Subsets of {0,1,2,3} in the order they are tried (gjk.cpp:120-135); the order
 * decides which sub-simplex is accepted first, so it is kept. */
static const int gjk_subsets[15] = {1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 12, 11, 13, 14, 15};
static const int gjk_tried[5] = {0, 0, 3, 7, 15};

static int popcount4(int s) { return (s & 1) + ((s >> 1) & 1) + ((s >> 2) & 1) + ((s >> 3) & 1); }

/* project(), gjk.cpp:302-414 */
static int gjk_project(gjk_point *w, int n, double *l, double *v) {
  double dots[4][4], dl[16][4], sum;
  if (n == 1) {
    l[0] = 1.0;
    v[0] = w[0].w[0]; v[1] = w[0].w[1]; v[2] = w[0].w[2];
    return 1;
  }
  for (int i = 0; i < n; ++i)
    for (int j = i; j < n; ++j) {
      dots[i][j] = dot3(w[i].w, w[j].w);
      dots[j][i] = dots[i][j];
    }
  for (int m = 0; m < gjk_tried[n]; ++m) {
    const int s = gjk_subsets[m];
    int ok = 1, k = 0;
    if (popcount4(s) == 1) {
      for (int i = 0; i < n; ++i)
        if (s & (1 << i)) { dl[s][i] = 1.0; k = i; break; }
      for (int j = 0; j < n; ++j)
        if (!(s & (1 << j))) {
          dl[s][j] = dots[k][k] - dots[k][j];
          if (dl[s][j] > 0.0) ok = 0;
        }
    } else {
      k = -1;
      for (int i = 0; i < n; ++i)
        if (s & (1 << i)) {
          const int o = s & ~(1 << i);
          if (k < 0) k = i;
          dl[s][i] = dl[o][i];
          if (dl[s][i] <= 0.0) ok = 0;
        }
      for (int j = 0; j < n; ++j)
        if (!(s & (1 << j))) {
          dl[s][j] = 0.0;
          for (int i = 0; i < n; ++i)
            if (s & (1 << i)) dl[s][j] += dl[s][i] * (dots[i][k] - dots[i][j]);
          if (dl[s][j] > 0.0) ok = 0;
        }
    }
    if (ok) {
      int o = 0;
      sum = 0.0;
      for (int i = 0; i < n; ++i)
        if (s & (1 << i)) {
          w[o] = w[i];
          l[o] = dl[s][i];
          sum += l[o];
          ++o;
        }
      v[0] = v[1] = v[2] = 0.0;
      for (int i = 0; i < o; ++i) {
        l[i] /= sum;
        v[0] = v[0] + l[i] * w[i].w[0];
        v[1] = v[1] + l[i] * w[i].w[1];
        v[2] = v[2] + l[i] * w[i].w[2];
      }
      return o;
    }
  }
  return 0;
}

/* minimal_support_point / maximal_support_point, gjk.cpp:141-165 (first extreme wins;
 * the first point is the fallback when every product is NaN). */
static const double *support_min(const double *c, int n, const double *v) {
  double best = DBL_MAX;
  const double *out = c;
  for (; n > 0; --n, c += 3) {
    const double dd = dot3(c, v);
    if (dd < best) { best = dd; out = c; }
  }
  return out;
}
static const double *support_max(const double *c, int n, const double *v) {
  double best = -DBL_MAX;
  const double *out = c;
  for (; n > 0; --n, c += 3) {
    const double dd = dot3(c, v);
    if (dd > best) { best = dd; out = c; }
  }
  return out;
}

/* gjk(a,na,b,nb,p,q), gjk.cpp:418-460; GEOMETRIC_EPSILON = 1e-6 (gjk.cpp:102) */
double dor_gjk(const double *a, int32_t na, const double *b, int32_t nb, double p[3], double q[3]) {
  const double GEPS = 1E-6;
  gjk_point w[4];
  double v[3], l[4], vlen, mi = 0.0;
  int toofar = 1, n = 0, j = 0;
  const int kmax = (na + nb) * (na + nb);
  v[0] = a[0] - b[0]; v[1] = a[1] - b[1]; v[2] = a[2] - b[2];
  vlen = sqrt(dot3(v, v));
  while (toofar && vlen > GEPS && n < 4 && j++ < kmax) {
    w[n].a = support_min(a, na, v);
    w[n].b = support_max(b, nb, v);
    for (int k = 0; k < 3; ++k) w[n].w[k] = w[n].a[k] - w[n].b[k];
    const double dlt = dot3(v, w[n].w) / vlen;
    mi = (mi > dlt) ? mi : dlt;
    toofar = (vlen - mi) > GEPS;
    if (toofar) {
      ++n;
      n = gjk_project(w, n, l, v);
      vlen = sqrt(dot3(v, v));
    }
  }
  if (n) {
    p[0] = p[1] = p[2] = 0.0;
    q[0] = q[1] = q[2] = 0.0;
    for (--n; n >= 0; --n)
      for (int k = 0; k < 3; ++k) {
        p[k] = p[k] + l[n] * w[n].a[k];
        q[k] = q[k] + l[n] * w[n].b[k];
      }
  } else {
    for (int k = 0; k < 3; ++k) { p[k] = a[k]; q[k] = b[k]; }
  }
  return vlen;
}

static void gjk_triangles(const double *xA, const double *yA, const double *zA,
                          const double *xB, const double *yB, const double *zB, double pq[6]) {
  double a[9], b[9];
  for (int v = 0; v < 3; ++v) {
    a[3 * v] = xA[v]; a[3 * v + 1] = yA[v]; a[3 * v + 2] = zA[v];
    b[3 * v] = xB[v]; b[3 * v + 1] = yB[v]; b[3 * v + 2] = zB[v];
  }
  dor_gjk(a, 3, b, 3, pq, pq + 3);
}

static inline double pq_distance(const double pq[6]) {
  /* d = |P_B - P_A| as written in bf.cpp:117 */
  return sqrt(((pq[3] - pq[0]) * (pq[3] - pq[0])) + ((pq[4] - pq[1]) * (pq[4] - pq[1])) +
              ((pq[5] - pq[2]) * (pq[5] - pq[2])));
}

/* ============================================================================
 * Pair list (ispc_bf / ispc_pen shape).
 * ========================================================================== */
static void pair_one(int32_t method, int64_t i, const double *a, const double *b, int64_t ld,
                     double max_error, double *p, double *q, double *dist, uint8_t *flags) {
  double xA[3], yA[3], zA[3], xB[3], yB[3], zB[3], pq[6];
  for (int v = 0; v < 3; ++v) {
    xA[v] = a[(3 * v + 0) * ld + i]; yA[v] = a[(3 * v + 1) * ld + i]; zA[v] = a[(3 * v + 2) * ld + i];
    xB[v] = b[(3 * v + 0) * ld + i]; yB[v] = b[(3 * v + 1) * ld + i]; zB[v] = b[(3 * v + 2) * ld + i];
  }
  int32_t flag = 0;
  switch (method) {
    case DOR_BF: dor_bf_solver(xA, yA, zA, xB, yB, zB, pq); break;
    case DOR_PENALTY: dor_penalty_solver(xA, yA, zA, xB, yB, zB, max_error, pq, &flag); break;
    case DOR_PENALTY_ITER: dor_penalty_solver_iter(xA, yA, zA, xB, yB, zB, max_error, pq, &flag); break;
    case DOR_GJK: gjk_triangles(xA, yA, zA, xB, yB, zB, pq); break;
    default: { /* per-pair hybrid: penalty, bf when the pair failed (hybrid.cpp:151-170 with nB=1) */
      dor_penalty_solver(xA, yA, zA, xB, yB, zB, max_error, pq, &flag);
      if (flag) dor_bf_solver(xA, yA, zA, xB, yB, zB, pq);
    }
  }
  for (int k = 0; k < 3; ++k) {
    p[k * ld + i] = pq[k];
    q[k * ld + i] = pq[3 + k];
  }
  dist[i] = pq_distance(pq);
  if (flags) flags[i] = (uint8_t)flag;
}

void dor_pairs(int32_t method, int64_t n, const double *a, const double *b, int64_t ld,
               double max_error, double *p, double *q, double *dist, uint8_t *flags,
               int32_t nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static) if (nthreads != 1)
#endif
  for (int64_t i = 0; i < n; ++i) pair_one(method, i, a, b, ld, max_error, p, q, dist, flags);
  (void)nthreads;
}

/* ============================================================================
 * contactpoint(PA, epsA, idA, QB, epsB, idB, friction), contactpoint.cpp:116-155
 * ========================================================================== */
void dor_make_contact(double xPA, double yPA, double zPA, double epsA, int32_t idA,
                      double xPB, double yPB, double zPB, double epsB, int32_t idB,
                      int32_t friction, dor_contact *c) {
  c->x[0] = (xPA + xPB) / 2.0;
  c->x[1] = (yPA + yPB) / 2.0;
  c->x[2] = (zPA + zPB) / 2.0;
  c->P[0] = xPA; c->P[1] = yPA; c->P[2] = zPA;
  c->Q[0] = xPB; c->Q[1] = yPB; c->Q[2] = zPB;
  c->eps_total = epsA + epsB;
  const double dist = sqrt(((c->Q[0] - c->P[0]) * (c->Q[0] - c->P[0])) + ((c->Q[1] - c->P[1]) * (c->Q[1] - c->P[1])) +
                           ((c->Q[2] - c->P[2]) * (c->Q[2] - c->P[2])));
  c->depth = (c->eps_total - dist);
  c->normal[0] = ((xPA - xPB) / dist);
  c->normal[1] = ((yPA - yPB) / dist);
  c->normal[2] = ((zPA - zPB) / dist);
  c->friction = friction;
  c->master = idA;
  c->slave = idB;
  c->penetration = 1;
  c->tri_a = -1;
  c->tri_b = -1;
}

/* ============================================================================
 * Particle-pair drivers (A-triangle rows, B-triangle columns, serial order).
 * ========================================================================== */
typedef struct {
  dor_contact *out;
  int64_t cap, n;
} contact_sink;

static void sink_push(contact_sink *s, const double pq[6], double epsA, int32_t idA, double epsB,
                      int32_t idB, int32_t fric, int32_t ta, int32_t tb) {
  if (s->n < s->cap) {
    dor_contact *c = &s->out[s->n];
    dor_make_contact(pq[0], pq[1], pq[2], epsA, idA, pq[3], pq[4], pq[5], epsB, idB, fric, c);
    c->tri_a = ta;
    c->tri_b = tb;
  }
  s->n++;
}

int64_t dor_detect(int32_t driver,
                   const double *xA, const double *yA, const double *zA, int32_t nA,
                   double epsA, int32_t fricA, int32_t idA,
                   const double *xB, const double *yB, const double *zB, int32_t nB,
                   double epsB, int32_t fricB, int32_t idB,
                   dor_contact *out, int64_t cap, dor_stats *stats) {
  contact_sink sink = {out, cap, 0};
  const double margin = epsA + epsB;
  const double max_err = (epsA + epsB) / 16; /* hybrid.cpp:60, penalty.cpp:86 */
  const int32_t fric = fricA && fricB;
  double *pq = (double *)malloc(sizeof(double) * 6 * (size_t)(nB > 0 ? nB : 1));
  double *d = (double *)malloc(sizeof(double) * (size_t)(nB > 0 ? nB : 1));
  int32_t *fl = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nB > 0 ? nB : 1));
  for (int32_t ta = 0; ta < nA; ++ta) {
    const int64_t iA = 3 * (int64_t)ta;
    const int use_penalty = driver == DOR_DRV_PENALTY || driver == DOR_DRV_HYBRID_BATCH ||
                            driver == DOR_DRV_HYBRID_TRIANGLE || driver == DOR_DRV_HYBRID_BATCH_STAT ||
                            driver == DOR_DRV_HYBRID_TRI_STAT;
    int32_t counter = 0;
    for (int32_t tb = 0; tb < nB; ++tb) {
      const int64_t iB = 3 * (int64_t)tb;
      fl[tb] = 0;
      if (driver == DOR_DRV_BF) {
        dor_bf_solver(xA + iA, yA + iA, zA + iA, xB + iB, yB + iB, zB + iB, pq + 6 * tb);
      } else if (driver == DOR_DRV_GJK) {
        gjk_triangles(xA + iA, yA + iA, zA + iA, xB + iB, yB + iB, zB + iB, pq + 6 * tb);
      } else if (driver == DOR_DRV_PENALTY_STAT) {
        int32_t it = 0; /* penalty.cpp:86 initialises the count to 0 */
        dor_penalty_solver_iter(xA + iA, yA + iA, zA + iA, xB + iB, yB + iB, zB + iB, max_err, pq + 6 * tb, &it);
        if (stats) stats->newton_hist[it]++;
      } else if (use_penalty) {
        dor_penalty_solver(xA + iA, yA + iA, zA + iA, xB + iB, yB + iB, zB + iB, max_err, pq + 6 * tb, &fl[tb]);
        counter += fl[tb] ? 1 : 0;
      }
      d[tb] = pq_distance(pq + 6 * tb);
    }
    /* fallback rules */
    int rerun = 0;
    if (driver == DOR_DRV_HYBRID_TRIANGLE) {
      rerun = counter > 0; /* hybrid.cpp:151-156 */
    } else if (driver == DOR_DRV_HYBRID_BATCH) {
      /* hybrid.cpp:434-440: counter*MaxErr > MaxErr*(3nB)/32 */
      rerun = (counter * max_err) > ((max_err * (double)(3 * (int64_t)nB)) / 32.0);
    } else if (driver == DOR_DRV_HYBRID_BATCH_STAT || driver == DOR_DRV_HYBRID_TRI_STAT) {
      /* hybrid.cpp:565-573 / 278-286: the bound uses the triangle count nB */
      rerun = (counter * max_err) > ((max_err * (double)nB) / 32);
      if (stats) {
        stats->batch_size += nB;
        stats->batch_error += max_err;
        stats->penalty_fails += counter;
        if (rerun) stats->batch_fails += 1;
      }
    }
    if (rerun)
      for (int32_t tb = 0; tb < nB; ++tb) {
        const int64_t iB = 3 * (int64_t)tb;
        dor_bf_solver(xA + iA, yA + iA, zA + iA, xB + iB, yB + iB, zB + iB, pq + 6 * tb);
        d[tb] = pq_distance(pq + 6 * tb);
      }
    /* contact rules */
    if (driver == DOR_DRV_HYBRID_BATCH_STAT || driver == DOR_DRV_HYBRID_TRI_STAT) {
      double minD = 1E99; /* hybrid.cpp:605-617: keep the row minimum only */
      for (int32_t tb = 0; tb < nB; ++tb) minD = (d[tb] < minD) ? d[tb] : minD;
      for (int32_t tb = 0; tb < nB; ++tb)
        if (d[tb] <= minD && d[tb] < margin) sink_push(&sink, pq + 6 * tb, epsA, idA, epsB, idB, fric, ta, tb);
    } else if (driver == DOR_DRV_PENALTY_STAT) {
      /* penalty.cpp:96: the contact loop runs over coordinate indices iB < nB, i.e. only
       * the first ceil(nB/3) triangles of B are checked (kept as written). */
      for (int32_t tb = 0; 3 * tb < nB; ++tb)
        if (d[tb] <= margin) sink_push(&sink, pq + 6 * tb, epsA, idA, epsB, idB, fric, ta, tb);
    } else if (driver == DOR_DRV_BF || driver == DOR_DRV_GJK) {
      for (int32_t tb = 0; tb < nB; ++tb) /* bf.cpp:125 uses <= */
        if (d[tb] <= margin) sink_push(&sink, pq + 6 * tb, epsA, idA, epsB, idB, fric, ta, tb);
    } else {
      for (int32_t tb = 0; tb < nB; ++tb) /* penalty.cpp:217, hybrid.cpp:176,466 use < */
        if (d[tb] < margin) sink_push(&sink, pq + 6 * tb, epsA, idA, epsB, idB, fric, ta, tb);
    }
  }
  free(pq);
  free(d);
  free(fl);
  return sink.n;
}

/* ============================================================================
 * Forces, forces.cpp:23-225 (spring, used part), 255-289 (friction), 291-396
 * (getContactsForces, mesh path).  normal_sign = -1 applies the inversion that
 * Collision::addCollision (Collision.cpp:176-184) stores for the second particle.
 * ========================================================================== */
void dor_contacts_forces(const dor_contact *cp, int64_t nc, double normal_sign,
                         const double posA[3], const double angA[3], const double linA[3], double massA,
                         const double posB[3], const double angB[3], const double linB[3], double massB,
                         const dor_material *mat, double force[3], double torque[3]) {
  for (int64_t k = 0; k < nc; ++k) {
    const dor_contact *c = &cp[k];
    double n[3];
    for (int i = 0; i < 3; ++i) n[i] = (normal_sign < 0) ? -1.0 * c->normal[i] : c->normal[i];
    double z[3], vi[3], vj[3], vij[3];
    z[0] = c->x[0] - posA[0]; z[1] = c->x[1] - posA[1]; z[2] = c->x[2] - posA[2];
    vi[0] = angA[1] * z[2] - angA[2] * z[1] + linA[0];
    vi[1] = angA[2] * z[0] - angA[0] * z[2] + linA[1];
    vi[2] = angA[0] * z[1] - angA[1] * z[0] + linA[2];
    z[0] = c->x[0] - posB[0]; z[1] = c->x[1] - posB[1]; z[2] = c->x[2] - posB[2];
    vj[0] = angB[1] * z[2] - angB[2] * z[1] + linB[0];
    vj[1] = angB[2] * z[0] - angB[0] * z[2] + linB[1];
    vj[2] = angB[0] * z[1] - angB[1] * z[0] + linB[2];
    vij[0] = vj[0] - vi[0]; vij[1] = vj[1] - vi[1]; vij[2] = vj[2] - vi[2];
    /* spring (forces.cpp:207-218) */
    const double ma = 1.0 / ((1.0 / massA) + (1.0 / massB));
    const double velocity = (vij[0] * n[0]) + (vij[1] * n[1]) + (vij[2] * n[2]);
    const double damp = mat->damper * 2.0 * sqrt(ma * mat->spring) * velocity;
    const double fmag = mat->spring * c->depth + damp;
    double f[3] = {fmag * n[0], fmag * n[1], fmag * n[2]};
    double fr[3] = {0.0, 0.0, 0.0};
    if (c->friction) { /* friction(): tangential part of vi, forces.cpp:265-289 */
      double vt[3];
      vt[0] = vi[0] - n[0] * ((vi[0] * n[0]) + (vi[1] * n[1]) + (vi[2] * n[2]));
      vt[1] = vi[1] - n[1] * ((vi[0] * n[0]) + (vi[1] * n[1]) + (vi[2] * n[2]));
      vt[2] = vi[2] - n[2] * ((vi[0] * n[0]) + (vi[1] * n[1]) + (vi[2] * n[2]));
      fr[0] = -vt[0] * mat->friction * fmag;
      fr[1] = -vt[1] * mat->friction * fmag;
      fr[2] = -vt[2] * mat->friction * fmag;
    }
    force[0] += f[0] + fr[0];
    force[1] += f[1] + fr[1];
    force[2] += f[2] + fr[2];
    double arm[3] = {c->x[0] - posA[0], c->x[1] - posA[1], c->x[2] - posA[2]};
    torque[0] += arm[1] * (f[2]) - arm[2] * (f[1]);
    torque[1] += arm[2] * (f[0]) - arm[0] * (f[2]);
    torque[2] += arm[0] * (f[1]) - arm[1] * (f[0]);
  }
}

/* ============================================================================
 * Dynamics, dynamics.cpp:26-242
 * ========================================================================== */
void dor_expmap(double O1, double O2, double O3, double L[9]) {
  const double v0 = O1 * O1, v1 = O2 * O2, v2 = O3 * O3;
  double angsq = v0 + v1 + v2, sx, cx;
  /* Taylor branch below 10 degrees (dynamics.cpp:38-63); coefficients as written there */
  if (angsq < 3.0461741978671E-02) {
    sx = 1.0 + (-1.666666666666667E-1 + (8.333333333333333E-3 + (-1.984126984126984E-4 +
         (2.755731922398589E-6 + (-2.505210838544172E-8 + 1.605904383682161E-10 * angsq) * angsq) * angsq) * angsq) * angsq) * angsq;
    cx = 0.5 + (-4.166666666666667E-2 + (1.388888888888889E-3 + (-2.480158730158730E-5 +
         (2.755731922398589E-7 + (-2.087675698786810E-9 + 1.147074559772972E-11 * angsq) * angsq) * angsq) * angsq) * angsq) * angsq;
  } else {
    const double t = angsq;
    angsq = sqrt(angsq);
    const double s = sin(angsq), c = cos(angsq);
    sx = s / angsq;
    cx = (1.0 - c) / t;
  }
  const double v01 = O1 * O2;
  const double v02 = O2 * O3; /* dynamics.cpp:78 computes Omega2*Omega3 here; kept */
  const double v12 = O2 * O3;
  const double s0 = sx * O1, s1 = sx * O2, s2 = sx * O3;
  L[0] = -cx * (v2 + v1);
  L[1] = cx * v01;
  L[2] = cx * v02;
  L[3] = L[1];
  L[4] = -cx * (v2 + v0);
  L[5] = cx * v12;
  L[6] = L[2];
  L[7] = L[5];
  L[8] = -cx * (v1 + v0);
  L[0] += 1.0;
  L[1] += s2;
  L[2] -= s1;
  L[3] -= s2;
  L[4] += 1.0;
  L[5] += s0;
  L[6] += s1;
  L[7] -= s0;
  L[8] += 1.0;
}

/* updateRotationMatrix, dynamics.cpp:104-138 */
void dor_update_rotation(double ang[3], const double W[3], double R[9], double step) {
  double DL[9], r[9];
  dor_expmap(step * W[0], step * W[1], step * W[2], DL);
  memcpy(r, R, sizeof r);
  for (int col = 0; col < 3; ++col)
    for (int row = 0; row < 3; ++row)
      R[3 * col + row] = r[row] * DL[3 * col] + r[3 + row] * DL[3 * col + 1] + r[6 + row] * DL[3 * col + 2];
  for (int row = 0; row < 3; ++row) ang[row] = R[row] * W[0] + R[3 + row] * W[1] + R[6 + row] * W[2];
}

/* updateAngular, dynamics.cpp:140-213 (eqs. 13-15) */
void dor_update_angular(double W[3], const double R[9], const double J[9], const double Ji[9],
                        const double tq[3], double step) {
  const double half = 0.5 * step;
  double T[3], DL[9], A[3], B[3];
  for (int i = 0; i < 3; ++i) T[i] = R[3 * i] * tq[0] + R[3 * i + 1] * tq[1] + R[3 * i + 2] * tq[2];
  dor_expmap(-half * W[0], -half * W[1], -half * W[2], DL);
  for (int i = 0; i < 3; ++i) A[i] = J[i] * W[0] + J[3 + i] * W[1] + J[6 + i] * W[2];
  for (int i = 0; i < 3; ++i) B[i] = DL[i] * A[0] + DL[3 + i] * A[1] + DL[6 + i] * A[2];
  for (int i = 0; i < 3; ++i) B[i] = B[i] + half * T[i];
  for (int i = 0; i < 3; ++i) A[i] = Ji[i] * B[0] + Ji[3 + i] * B[1] + Ji[6 + i] * B[2];
  for (int i = 0; i < 3; ++i) B[i] = J[i] * A[0] + J[3 + i] * A[1] + J[6 + i] * A[2];
  T[0] -= A[1] * B[2] - A[2] * B[1];
  T[1] -= A[2] * B[0] - A[0] * B[2];
  T[2] -= A[0] * B[1] - A[1] * B[0];
  T[0] *= step; T[1] *= step; T[2] *= step;
  for (int i = 0; i < 3; ++i) W[i] = W[i] + Ji[i] * T[0] + Ji[3 + i] * T[1] + Ji[6 + i] * T[2];
}

/* updateVertices, dynamics.cpp:215-242 */
void dor_update_vertex(double *x, double *y, double *z, double rx, double ry, double rz,
                       const double R[9], const double pos[3], const double ref_pos[3]) {
  const double C0 = rx - ref_pos[0], C1 = ry - ref_pos[1], C2 = rz - ref_pos[2];
  *x = pos[0] + (R[0] * C0 + R[3] * C1 + R[6] * C2);
  *y = pos[1] + (R[1] * C0 + R[4] * C1 + R[7] * C2);
  *z = pos[2] + (R[2] * C0 + R[5] * C1 + R[8] * C2);
}

/* ============================================================================
 * Whole time step in the multiscale update order (Collision.cpp:1043-1127 forces
 * from the previous traversal's contacts; MoveParticles.cpp:63-112 move;
 * Collision.cpp:301-660 detection; Collision.cpp:988-1008 swap).  Candidate pairs
 * are body pairs (i<j, not both obstacles) whose bounding spheres grown by the
 * epsilons overlap; triangle pairs whose bounding boxes are farther apart than
 * epsA+epsB cannot hold a bf() contact and are skipped.  Body i is A, j is B.
 * ========================================================================== */
struct dor_sim {
  dor_contact *c;
  int64_t n, cap;
};

dor_sim *dor_sim_create(void) { return (dor_sim *)calloc(1, sizeof(dor_sim)); }
void dor_sim_destroy(dor_sim *s) {
  if (s) { free(s->c); free(s); }
}

static void sim_push(dor_sim *s, const dor_contact *c) {
  if (s->n == s->cap) {
    s->cap = s->cap ? 2 * s->cap : 1024;
    s->c = (dor_contact *)realloc(s->c, sizeof(dor_contact) * (size_t)s->cap);
  }
  s->c[s->n++] = *c;
}

static void tri_box(const dor_scene *sc, int64_t t, double lo[3], double hi[3]) {
  const double *cs[3] = {sc->x, sc->y, sc->z};
  for (int k = 0; k < 3; ++k) {
    double a = cs[k][3 * t], b = cs[k][3 * t + 1], c = cs[k][3 * t + 2];
    lo[k] = a < b ? (a < c ? a : c) : (b < c ? b : c);
    hi[k] = a > b ? (a > c ? a : c) : (b > c ? b : c);
  }
}

static void sim_detect(dor_sim *s, const dor_scene *sc) {
  s->n = 0;
  const int32_t nb = sc->n_bodies;
  for (int32_t i = 0; i < nb; ++i)
    for (int32_t j = i + 1; j < nb; ++j) {
      if (sc->obstacle[i] && sc->obstacle[j]) continue;
      const double dx = sc->pos[3 * j] - sc->pos[3 * i], dy = sc->pos[3 * j + 1] - sc->pos[3 * i + 1],
                   dz = sc->pos[3 * j + 2] - sc->pos[3 * i + 2];
      const double reach = sc->radius[i] + sc->radius[j] + sc->eps[i] + sc->eps[j];
      if (dx * dx + dy * dy + dz * dz > reach * reach * (1.0 + 1e-9) + 1e-18) continue;
      const double margin = sc->eps[i] + sc->eps[j];
      const double cull = margin * (1.0 + 1e-9) + 1e-12;
      const int32_t fric = sc->friction[i] && sc->friction[j];
      for (int64_t ta = sc->tri_offset[i]; ta < sc->tri_offset[i + 1]; ++ta) {
        double alo[3], ahi[3];
        tri_box(sc, ta, alo, ahi);
        for (int64_t tb = sc->tri_offset[j]; tb < sc->tri_offset[j + 1]; ++tb) {
          double blo[3], bhi[3], g2 = 0.0;
          tri_box(sc, tb, blo, bhi);
          for (int k = 0; k < 3; ++k) {
            double g = blo[k] - ahi[k];
            const double g2k = alo[k] - bhi[k];
            if (g2k > g) g = g2k;
            if (g > 0) g2 += g * g;
          }
          if (g2 > cull * cull) continue;
          double pq[6];
          dor_bf_solver(sc->x + 3 * ta, sc->y + 3 * ta, sc->z + 3 * ta, sc->x + 3 * tb, sc->y + 3 * tb,
                        sc->z + 3 * tb, pq);
          if (pq_distance(pq) <= margin) {
            dor_contact c;
            dor_make_contact(pq[0], pq[1], pq[2], sc->eps[i], i, pq[3], pq[4], pq[5], sc->eps[j], j, fric, &c);
            c.tri_a = (int32_t)(ta - sc->tri_offset[i]);
            c.tri_b = (int32_t)(tb - sc->tri_offset[j]);
            sim_push(s, &c);
          }
        }
      }
    }
}

int64_t dor_sim_run(dor_sim *s, dor_scene *sc, const dor_step_params *prm, int32_t nsteps,
                    int64_t *contacts_per_step) {
  const int32_t nb = sc->n_bodies;
  double *F = (double *)malloc(sizeof(double) * 3 * (size_t)nb);
  double *T = (double *)malloc(sizeof(double) * 3 * (size_t)nb);
  uint8_t *has = (uint8_t *)malloc((size_t)nb);
  const double dt = prm->dt;
  for (int32_t step = 0; step < nsteps; ++step) {
    /* 1. forces from the contacts of the previous detection; every body reads the
     *    end-of-previous-step state of itself and of its partner (the partner copy
     *    stored at detection time, Collision.cpp:163-166). */
    memset(F, 0, sizeof(double) * 3 * (size_t)nb);
    memset(T, 0, sizeof(double) * 3 * (size_t)nb);
    memset(has, 0, (size_t)nb);
    /* gather per body its partner list in ascending partner order */
    for (int32_t i = 0; i < nb; ++i) {
      if (sc->obstacle[i]) continue;
      /* partners j < i: pairs (j,i) where i is slave; partners j > i: pairs (i,j) */
      for (int32_t j = 0; j < nb; ++j) {
        if (j == i) continue;
        const int32_t m = i < j ? i : j, sl = i < j ? j : i;
        int64_t first = -1, count = 0;
        /* contacts are sorted by (master, slave): binary search the block */
        int64_t lo = 0, hi = s->n;
        while (lo < hi) {
          const int64_t mid = (lo + hi) / 2;
          const dor_contact *c = &s->c[mid];
          if (c->master < m || (c->master == m && c->slave < sl)) lo = mid + 1;
          else hi = mid;
        }
        for (int64_t k = lo; k < s->n && s->c[k].master == m && s->c[k].slave == sl; ++k) {
          if (first < 0) first = k;
          ++count;
        }
        if (count == 0) continue;
        has[i] = 1;
        double rf[3] = {0, 0, 0}, rt[3] = {0, 0, 0};
        dor_contacts_forces(s->c + first, count, i < j ? 1.0 : -1.0, sc->pos + 3 * i, sc->ang + 3 * i,
                            sc->vel + 3 * i, sc->mass[i], sc->pos + 3 * j, sc->ang + 3 * j, sc->vel + 3 * j,
                            sc->mass[j], &prm->mat, rf, rt);
        F[3 * i] += rf[0]; F[3 * i + 1] += rf[1]; F[3 * i + 2] += rf[2];
        T[3 * i] += rt[0]; T[3 * i + 1] += rt[1]; T[3 * i + 2] += rt[2];
      }
    }
    for (int32_t i = 0; i < nb; ++i) {
      if (!has[i]) continue;
      for (int k = 0; k < 3; ++k) sc->vel[3 * i + k] += dt * (F[3 * i + k] / sc->mass[i]);
      dor_update_angular(sc->ref_ang + 3 * i, sc->rot + 9 * i, sc->inertia + 9 * i, sc->inverse + 9 * i,
                         T + 3 * i, dt);
    }
    /* 2. move (MoveParticles.cpp:63-112) */
    for (int32_t i = 0; i < nb; ++i) {
      if (sc->obstacle[i]) continue;
      for (int k = 0; k < 3; ++k) sc->vel[3 * i + k] += dt * (prm->gravity[k]);
      for (int k = 0; k < 3; ++k) sc->pos[3 * i + k] += dt * sc->vel[3 * i + k];
      dor_update_rotation(sc->ang + 3 * i, sc->ref_ang + 3 * i, sc->rot + 9 * i, dt);
      for (int64_t v = 3 * sc->tri_offset[i]; v < 3 * sc->tri_offset[i + 1]; ++v)
        dor_update_vertex(&sc->x[v], &sc->y[v], &sc->z[v], sc->rx[v], sc->ry[v], sc->rz[v], sc->rot + 9 * i,
                          sc->pos + 3 * i, sc->ref_pos + 3 * i);
    }
    /* 3. detection; contacts come out sorted by (master, slave, tri_a, tri_b) */
    sim_detect(s, sc);
    if (contacts_per_step) contacts_per_step[step] = s->n;
  }
  free(F);
  free(T);
  free(has);
  return s->n;
}

int64_t dor_sim_contacts(const dor_sim *s, dor_contact *out, int64_t cap) {
  const int64_t n = s->n < cap ? s->n : cap;
  if (n > 0) memcpy(out, s->c, sizeof(dor_contact) * (size_t)n);
  return s->n;
}

/* ---- contact de-duplication: filter.cpp --------------------------------------------- */

static int dor_near(const double *x, int64_t ld, int64_t i, const double *y, int64_t ldy, int64_t j, double eps) {
  /* filter.cpp:16-21 / 92-97: the three coordinate differences, each |.| < eps */
  return fabs(x[i] - y[j]) < eps && fabs(x[ld + i] - y[ldy + j]) < eps &&
         fabs(x[2 * ld + i] - y[2 * ldy + j]) < eps;
}

void dor_filter_new(int64_t n, const double *x, int64_t ld, const int32_t *master, const int32_t *slave,
                    double eps, uint8_t *keep) {
  int64_t s = 0;
  while (s < n) {
    int64_t e = s + 1;
    while (e < n && master[e] == master[s] && slave[e] == slave[s]) ++e;
    /* filter.cpp:80-101: a contact survives unless a survivor before it is near */
    for (int64_t i = s; i < e; ++i) {
      int hit = 0;
      for (int64_t j = s; j < i && !hit; ++j)
        if (keep[j] && dor_near(x, ld, i, x, ld, j, eps)) hit = 1;
      keep[i] = hit ? 0 : 1;
    }
    s = e;
  }
}

void dor_filter_old(int64_t ns, const double *xs, int64_t lds, const int32_t *ms, const int32_t *ss, int64_t nn,
                    const double *xn, int64_t ldn, const int32_t *mn, const int32_t *sn, double eps,
                    uint8_t *keep) {
  for (int64_t i = 0; i < nn; ++i) {
    int hit = 0;
    for (int64_t j = 0; j < ns && !hit; ++j)
      if (ms[j] == mn[i] && ss[j] == sn[i] && dor_near(xn, ldn, i, xs, lds, j, eps)) hit = 1;
    keep[i] = hit ? 0 : 1;
  }
}

/* ---- sphere model: point.cpp, sphere.cpp --------------------------------------------- */

#define DOR_DOT(a, b) ((a)[0] * (b)[0] + (a)[1] * (b)[1] + (a)[2] * (b)[2])

double dor_pt(const double TP1[3], const double TP2[3], const double TP3[3], const double c[3], double tq[3]) {
  double E0[3], E1[3], D[3];
  for (int k = 0; k < 3; ++k) {
    E0[k] = TP2[k] - TP1[k];
    E1[k] = TP3[k] - TP1[k];
    D[k] = TP1[k] - c[k];
  }
  const double a = DOR_DOT(E0, E0), b = DOR_DOT(E0, E1), cc = DOR_DOT(E1, E1);
  const double d = DOR_DOT(E0, D), e = DOR_DOT(E1, D), f = DOR_DOT(D, D);
  const double det = a * cc - b * b;
  double s = b * e - cc * d, t = b * d - a * e, sq = 0;
  /* the seven regions of point.cpp:41-203 */
  if ((s + t) <= det) {
    if (s < 0) {
      if (t < 0) { /* region 4 */
        if (d < 0) {
          t = 0;
          if (-d >= a) { s = 1; sq = a + 2 * d + f; }
          else { s = -d / a; sq = d * s + f; }
        } else {
          s = 0;
          if (e >= 0) { t = 0; sq = f; }
          else if (-e >= cc) { t = 1; sq = cc + 2 * e + f; }
          else { t = -e / cc; sq = e * t + f; }
        }
      } else { /* region 3 */
        s = 0;
        if (e >= 0) { t = 0; sq = f; }
        else if (-e >= cc) { t = 1; sq = cc + 2 * e + f; }
        else { t = -e / cc; sq = e * t + f; }
      }
    } else if (t < 0) { /* region 5 */
      t = 0;
      if (d >= 0) { s = 0; sq = f; }
      else if (-d >= a) { s = 1; sq = a + 2 * d + f; }
      else { s = -d / a; sq = d * s + f; }
    } else { /* region 0 */
      const double inv = 1 / det;
      s = s * inv;
      t = t * inv;
      sq = s * (a * s + b * t + 2 * d) + t * (b * s + cc * t + 2 * e) + f;
    }
  } else {
    if (s < 0) { /* region 2 */
      const double tmp0 = b + d, tmp1 = cc + e;
      if (tmp1 > tmp0) {
        const double numer = tmp1 - tmp0, denom = a - 2 * b + cc;
        if (numer >= denom) { s = 1; t = 0; sq = a + 2 * d + f; }
        else { s = numer / denom; t = 1 - s; sq = s * (a * s + b * t + 2 * d) + t * (b * s + cc * t + 2 * e) + f; }
      } else {
        s = 0;
        if (tmp1 <= 0) { t = 1; sq = cc + 2 * e + f; }
        else if (e >= 0) { t = 0; sq = f; }
        else { t = -e / cc; sq = e * t + f; }
      }
    } else if (t < 0) { /* region 6 */
      const double tmp0 = b + e, tmp1 = a + d;
      if (tmp1 > tmp0) {
        const double numer = tmp1 - tmp0, denom = a - 2 * b + cc;
        if (numer >= denom) { t = 1; s = 0; sq = cc + 2 * e + f; }
        else { t = numer / denom; s = 1 - t; sq = s * (a * s + b * t + 2 * d) + t * (b * s + cc * t + 2 * e) + f; }
      } else {
        t = 0;
        if (tmp1 <= 0) { s = 1; sq = a + 2 * d + f; }
        else if (d >= 0) { s = 0; sq = f; }
        else { s = -d / a; sq = d * s + f; }
      }
    } else { /* region 1 */
      const double numer = cc + e - b - d;
      if (numer <= 0) { s = 0; t = 1; sq = cc + 2 * e + f; }
      else {
        const double denom = a - 2 * b + cc;
        if (numer >= denom) { s = 1; t = 0; sq = a + 2 * d + f; }
        else { s = numer / denom; t = 1 - s; sq = s * (a * s + b * t + 2 * d) + t * (b * s + cc * t + 2 * e) + f; }
      }
    }
  }
  if (sq < 0) sq = 0;
  for (int k = 0; k < 3; ++k) tq[k] = TP1[k] + (E1[k] * t) + (E0[k] * s);
  return sqrt(sq);
}

static double dor_contact_distance(const dor_contact *c) {
  return sqrt(((c->Q[0] - c->P[0]) * (c->Q[0] - c->P[0])) + ((c->Q[1] - c->P[1]) * (c->Q[1] - c->P[1])) +
              ((c->Q[2] - c->P[2]) * (c->Q[2] - c->P[2])));
}

int64_t dor_sphere(const double cA[3], double dA, double epsA, int32_t fricA, int32_t idA, const double cB[3],
                   double dB, double epsB, int32_t fricB, int32_t idB, dor_contact *out) {
  /* sphere.cpp:46-76 */
  const double distance = sqrt(((cB[0] - cA[0]) * (cB[0] - cA[0])) + ((cB[1] - cA[1]) * (cB[1] - cA[1])) +
                               ((cB[2] - cA[2]) * (cB[2] - cA[2])));
  double n[3], PA[3], PB[3];
  for (int k = 0; k < 3; ++k) n[k] = (1.0 / distance) * (cB[k] - cA[k]);
  for (int k = 0; k < 3; ++k) {
    PA[k] = cA[k] + ((dA / 2) * n[k]);
    PB[k] = cB[k] - ((dB / 2) * n[k]);
  }
  dor_contact c;
  dor_make_contact(PA[0], PA[1], PA[2], epsA, idA, PB[0], PB[1], PB[2], epsB, idB, (fricA & fricB) ? 1 : 0, &c);
  if (dor_contact_distance(&c) <= (epsA + epsB)) {
    if (out) *out = c;
    return 1;
  }
  return 0;
}

int64_t dor_sphere_mesh(int32_t ba, const double c[3], double d, double epsS, int32_t fricS, int32_t idS,
                        const double *x, const double *y, const double *z, int32_t nT, double epsM, int32_t fricM,
                        int32_t idM, dor_contact *out, int64_t cap) {
  int64_t n = 0;
  for (int32_t i = 0; i < 3 * nT; i += 3) {
    const double TP1[3] = {x[i], y[i], z[i]}, TP2[3] = {x[i + 1], y[i + 1], z[i + 1]},
                 TP3[3] = {x[i + 2], y[i + 2], z[i + 2]};
    double Q[3], S[3];
    /* sphere.cpp:112-124 / 175-187 */
    const double distance = dor_pt(TP1, TP2, TP3, c, Q) - (d / 2.0);
    for (int k = 0; k < 3; ++k) {
      const double nk = (Q[k] - c[k]) / (distance + (d / 2.0));
      S[k] = c[k] + ((d / 2.0) * nk);
    }
    dor_contact ct;
    const int32_t fr = (fricS & fricM) ? 1 : 0;
    if (ba == 0)
      dor_make_contact(S[0], S[1], S[2], epsS, idS, Q[0], Q[1], Q[2], epsM, idM, fr, &ct);
    else /* sphere.cpp:189: the mesh point first, with the sphere's epsilon and id */
      dor_make_contact(Q[0], Q[1], Q[2], epsS, idS, S[0], S[1], S[2], epsM, idM, fr, &ct);
    if (dor_contact_distance(&ct) <= (epsS + epsM)) {
      if (out && n < cap) {
        out[n] = ct;
        out[n].tri_b = i / 3;
      }
      ++n;
    }
  }
  return n;
}

int32_t dor_sphere_overlay(const double cA[3], double rA, const double cB[3], double rB) {
  const double distance = sqrt(pow(cB[0] - cA[0], 2) + pow(cB[1] - cA[1], 2) + pow(cB[2] - cA[2], 2));
  return distance <= rA + rB ? 1 : 0;
}
