// tri_cert.cuh -- bfSolver's result computed with an FP32 filter and FP64 finishing.
//
// bfSolver (bf.cpp:217-1178) returns the minimum over 15 features (9 edge-edge, 6
// vertex-face) with fixed tie rules.  Here every feature is first evaluated in FP32 in a
// frame centred on A's first vertex: the FP32 value is the length of an explicit point
// pair lying on the two features, so it can overestimate the feature's distance (a
// poorly conditioned parameter) but can underestimate it only by rounding, by less than
// the band
//     eps = L * (64 u32 + 4 sqrt(16 u64)),  L = extent of the pair's bounding box,
// which also covers the reference's own FP64 rounding (its vertex-face distance comes
// from a quadratic form whose error grows like sqrt(u64) * L near contact).
// The feature with the smallest FP32 value is then evaluated in FP64 with the reference's
// arithmetic; its value `best` bounds the reference minimum from above.  Every feature
// whose lower bound d32 - eps does not exceed `best` is evaluated in FP64 too, and the
// reference's selection rule is applied to these candidates in the reference's order.
// All features that attain the reference minimum are candidates, so the selected feature,
// and the closest points computed from it in FP64, equal bfSolver's bit for bit.
#pragma once
#include "tri_ref.cuh"

namespace delta {

// FP32 edge-edge: Sunday's clamp in float, then the explicit point pair.
__device__ __forceinline__ float seg_seg_f32(const float *HA, const float *TA, const float *HB, const float *TB) {
  float u[3], v[3], w[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    u[k] = HA[k] - TA[k];
    v[k] = HB[k] - TB[k];
    w[k] = TA[k] - TB[k];
  }
  const float a = dot3(u, u), b = dot3(u, v), c = dot3(v, v), d = dot3(u, w), e = dot3(v, w);
  const float D = a * c - b * b;
  float sN, sD = D, tN, tD = D;
  if (D <= 1e-30f * (a * c)) {  // parallel in FP32
    sN = 0.f; sD = 1.f; tN = e; tD = c;
  } else {
    sN = b * e - c * d;
    tN = a * e - b * d;
    if (sN < 0.f) { sN = 0.f; tN = e; tD = c; }
    else if (sN > sD) { sN = sD; tN = e + b; tD = c; }
  }
  if (tN < 0.f) {
    tN = 0.f;
    if (-d < 0.f) sN = 0.f;
    else if (-d > a) sN = sD;
    else { sN = -d; sD = a; }
  } else if (tN > tD) {
    tN = tD;
    if ((-d + b) < 0.f) sN = 0.f;
    else if ((-d + b) > a) sN = sD;
    else { sN = -d + b; sD = a; }
  }
  const float sc = fminf(fmaxf(sD != 0.f ? sN / sD : 0.f, 0.f), 1.f);
  const float tc = fminf(fmaxf(tD != 0.f ? tN / tD : 0.f, 0.f), 1.f);
  float r[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) r[k] = (TA[k] + sc * u[k]) - (TB[k] + tc * v[k]);
  return sqrtf(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
}

// FP32 vertex-face: Eberly's region choice in float for (s, t), then the explicit
// point V0 + s E0 + t E1 and its distance to X.
__device__ __forceinline__ float pt_tri_f32(const float *V0, const float *V1, const float *V2, const float *X) {
  float E0[3], E1[3], Dv[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    E0[k] = V1[k] - V0[k];
    E1[k] = V2[k] - V0[k];
    Dv[k] = V0[k] - X[k];
  }
  const float a = dot3(E0, E0), b = dot3(E0, E1), c = dot3(E1, E1), d = dot3(E0, Dv), e = dot3(E1, Dv);
  const float det = a * c - b * b;
  float s = b * e - c * d, t = b * d - a * e;
  if (s + t <= det) {
    if (s < 0.f) {
      if (t < 0.f) {
        if (d < 0.f) { t = 0.f; s = (-d >= a) ? 1.f : -d / a; }
        else { s = 0.f; t = (e >= 0.f) ? 0.f : ((-e >= c) ? 1.f : -e / c); }
      } else { s = 0.f; t = (e >= 0.f) ? 0.f : ((-e >= c) ? 1.f : -e / c); }
    } else if (t < 0.f) { t = 0.f; s = (d >= 0.f) ? 0.f : ((-d >= a) ? 1.f : -d / a); }
    else { const float inv = 1.f / det; s *= inv; t *= inv; }
  } else {
    if (s < 0.f) {
      const float tmp0 = b + d, tmp1 = c + e;
      if (tmp1 > tmp0) {
        const float numer = tmp1 - tmp0, denom = a - 2.f * b + c;
        s = (numer >= denom) ? 1.f : numer / denom;
        t = 1.f - s;
      } else { s = 0.f; t = (tmp1 <= 0.f) ? 1.f : ((e >= 0.f) ? 0.f : -e / c); }
    } else if (t < 0.f) {
      const float tmp0 = b + e, tmp1 = a + d;
      if (tmp1 > tmp0) {
        const float numer = tmp1 - tmp0, denom = a - 2.f * b + c;
        t = (numer >= denom) ? 1.f : numer / denom;
        s = 1.f - t;
      } else { t = 0.f; s = (tmp1 <= 0.f) ? 1.f : ((d >= 0.f) ? 0.f : -d / a); }
    } else {
      const float numer = c + e - b - d, denom = a - 2.f * b + c;
      s = (numer <= 0.f) ? 0.f : ((numer >= denom) ? 1.f : numer / denom);
      t = 1.f - s;
    }
  }
  float r[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) r[k] = (V0[k] + s * E0[k] + t * E1[k]) - X[k];
  return sqrtf(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
}

// Relative band per unit of bounding-box extent: 64 u32 + 4 sqrt(16 u64).
constexpr double kCertBand = 64.0 * 5.9604644775390625e-08 + 4.0 * 4.2146848510894035e-08;

// Returns bfSolver's closest points (pq, FP64) and the number of FP64 feature evaluations.
__device__ __forceinline__ int bf_cert(const double A64[3][3], const double B64[3][3], double pq_out[6]) {
  float A[3][3], B[3][3];
  double lo[3], hi[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    lo[k] = hi[k] = A64[0][k];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      A[v][k] = (float)(A64[v][k] - A64[0][k]);
      B[v][k] = (float)(B64[v][k] - A64[0][k]);
      lo[k] = fmin(lo[k], fmin(A64[v][k], B64[v][k]));
      hi[k] = fmax(hi[k], fmax(A64[v][k], B64[v][k]));
    }
  }
  const double L = fmax(hi[0] - lo[0], fmax(hi[1] - lo[1], hi[2] - lo[2]));
  const double eps = L * kCertBand;

  float d32[15];
#pragma unroll
  for (int j = 0; j < 9; ++j) d32[j] = seg_seg_f32(A[j / 3], A[(j / 3 + 1) % 3], B[j % 3], B[(j % 3 + 1) % 3]);
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    d32[9 + j] = pt_tri_f32(A[0], A[1], A[2], B[j]);
    d32[12 + j] = pt_tri_f32(B[0], B[1], B[2], A[j]);
  }
  int fmin_ = 0;
  float dmin = d32[0];
#pragma unroll
  for (int f = 1; f < 15; ++f)
    if (d32[f] < dmin) { dmin = d32[f]; fmin_ = f; }

  xf64 Ax[3][3], Bx[3][3];
#pragma unroll
  for (int v = 0; v < 3; ++v)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      Ax[v][k] = xf64(A64[v][k]);
      Bx[v][k] = xf64(B64[v][k]);
    }
  xf64 c0, c1;
  const xf64 best = feature_ref(Ax, Bx, fmin_, c0, c1);
  int evals = 1;

  xf64 ssmin = xf64(1E+30), ssc = xf64(0.0), ttc = xf64(0.0), ptmin = xf64(1E30), ss = xf64(0.0), tt = xf64(0.0);
  int ssid = 0, id = 0;
#pragma unroll
  for (int f = 0; f < 15; ++f) {
    // NaN in either value keeps the feature (the comparison is false)
    const bool cand = !((double)d32[f] - eps > best.v);
    if (cand) {
      xf64 p0, p1, dist;
      if (f == fmin_) { dist = best; p0 = c0; p1 = c1; }
      else { dist = feature_ref(Ax, Bx, f, p0, p1); ++evals; }
      if (f < 9) {
        if (dist < ssmin) { ssmin = dist; ssc = p0; ttc = p1; ssid = f; }
      } else {
        if (dist < ptmin) { ptmin = dist; ss = p0; tt = p1; id = f - 9; }
      }
    }
  }
  xf64 pq[6];
  if (ptmin > ssmin) seg_seg_points(Ax, Bx, ssid, ssc, ttc, pq);
  else pt_tri_points(Ax, Bx, id, ss, tt, pq);
#pragma unroll
  for (int k = 0; k < 6; ++k) pq_out[k] = pq[k].v;
  return evals;
}

}  // namespace delta
