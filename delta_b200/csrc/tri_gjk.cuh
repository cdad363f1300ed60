// tri_gjk.cuh -- GJK distance between two triangles with Johnson's sub-simplex
// projection, the arithmetic of gjk.cpp:302-460 (Solfec's gjk) for na = nb = 3.
#pragma once
#include "real.cuh"

namespace delta {

// Simplex vertex: Minkowski point w = A[ia] - B[ib].
template <class R>
struct GjkVertex {
  R w[3];
  int ia, ib;
};

// project(), gjk.cpp:302-414.  Subsets are tried in the order of gjk.cpp:120-135
// (the order decides which sub-simplex is accepted first).
template <class R>
__device__ __forceinline__ int gjk_project(GjkVertex<R> *w, int n, R *l, R *v) {
  constexpr int subsets[15] = {1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 12, 11, 13, 14, 15};
  constexpr int tried[5] = {0, 0, 3, 7, 15};
  if (n == 1) {
    l[0] = R(1.0);
    v[0] = w[0].w[0]; v[1] = w[0].w[1]; v[2] = w[0].w[2];
    return 1;
  }
  R dots[4][4], dl[16][4];
  for (int i = 0; i < n; ++i)
    for (int j = i; j < n; ++j) {
      dots[i][j] = dot3(w[i].w, w[j].w);
      dots[j][i] = dots[i][j];
    }
  for (int m = 0; m < tried[n]; ++m) {
    const int s = subsets[m];
    const int card = __popc(s);
    bool ok = true;
    int k = 0;
    if (card == 1) {
      k = __ffs(s) - 1;
      dl[s][k] = R(1.0);
      for (int j = 0; j < n; ++j)
        if (!(s & (1 << j))) {
          dl[s][j] = dots[k][k] - dots[k][j];
          if (dl[s][j] > R(0.0)) ok = false;
        }
    } else {
      k = -1;
      for (int i = 0; i < n; ++i)
        if (s & (1 << i)) {
          const int o = s & ~(1 << i);
          if (k < 0) k = i;
          dl[s][i] = dl[o][i];
          if (dl[s][i] <= R(0.0)) ok = false;
        }
      for (int j = 0; j < n; ++j)
        if (!(s & (1 << j))) {
          dl[s][j] = R(0.0);
          for (int i = 0; i < n; ++i)
            if (s & (1 << i)) dl[s][j] += dl[s][i] * (dots[i][k] - dots[i][j]);
          if (dl[s][j] > R(0.0)) ok = false;
        }
    }
    if (ok) {
      int o = 0;
      R sum = R(0.0);
      for (int i = 0; i < n; ++i)
        if (s & (1 << i)) {
          w[o] = w[i];
          l[o] = dl[s][i];
          sum += l[o];
          ++o;
        }
      v[0] = v[1] = v[2] = R(0.0);
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

// gjk(a,3,b,3,p,q), gjk.cpp:418-460; GEOMETRIC_EPSILON = 1e-6 (gjk.cpp:102).  The
// support points are the first extreme vertex (gjk.cpp:141-165).
template <class R>
__device__ __forceinline__ R gjk_ref(const R A[3][3], const R B[3][3], R pq[6]) {
  const R GEPS = R(1E-6);
  GjkVertex<R> w[4];
  R v[3], l[4], mi = R(0.0);
  bool toofar = true;
  int n = 0, j = 0;
  const int kmax = 36;
#pragma unroll
  for (int k = 0; k < 3; ++k) v[k] = A[0][k] - B[0][k];
  R vlen = sqrt_(dot3(v, v));
  while (toofar && vlen > GEPS && n < 4 && j++ < kmax) {
    int ia = 0, ib = 0;
    R best = R(1.7976931348623157e308);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const R dd = dot3(A[q], v);
      if (dd < best) { best = dd; ia = q; }
    }
    best = R(-1.7976931348623157e308);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const R dd = dot3(B[q], v);
      if (dd > best) { best = dd; ib = q; }
    }
    R wa[3], wb[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      wa[k] = ia == 0 ? A[0][k] : (ia == 1 ? A[1][k] : A[2][k]);
      wb[k] = ib == 0 ? B[0][k] : (ib == 1 ? B[1][k] : B[2][k]);
    }
    w[n].ia = ia;
    w[n].ib = ib;
#pragma unroll
    for (int k = 0; k < 3; ++k) w[n].w[k] = wa[k] - wb[k];
    const R dlt = dot3(v, w[n].w) / vlen;
    mi = (mi > dlt) ? mi : dlt;
    toofar = (vlen - mi) > GEPS;
    if (toofar) {
      ++n;
      n = gjk_project(w, n, l, v);
      vlen = sqrt_(dot3(v, v));
    }
  }
  if (n) {
#pragma unroll
    for (int k = 0; k < 6; ++k) pq[k] = R(0.0);
    for (--n; n >= 0; --n) {
      const int ia = w[n].ia, ib = w[n].ib;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const R av = ia == 0 ? A[0][k] : (ia == 1 ? A[1][k] : A[2][k]);
        const R bv = ib == 0 ? B[0][k] : (ib == 1 ? B[1][k] : B[2][k]);
        pq[k] = pq[k] + l[n] * av;
        pq[3 + k] = pq[3 + k] + l[n] * bv;
      }
    }
  } else {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      pq[k] = A[0][k];
      pq[3 + k] = B[0][k];
    }
  }
  return vlen;
}

}  // namespace delta
