// zoltan_shim.cpp -- extern "C" entry points over the reference's zoltan/ narrowphase
// (zoltan/bf.cpp, penalty.cpp, hybrid.cpp, compiled where they lie by oracle/Makefile).
// TEST INFRASTRUCTURE ONLY: the pin of the zoltan part of the restatement
// (zoltan_oracle.c).  Layouts as in zoltan_oracle.c: d, e, f, p, q are 3 planes of ld
// doubles.
#include <cstdint>

// zoltan/bf.cpp:26, zoltan/penalty.h:47-50, zoltan/hybrid.cpp:37-40
void bf(double xA[3], double yA[3], double zA[3], double xB[3], double yB[3], double zB[3], double &xPA, double &yPA,
        double &zPA, double &xPB, double &yPB, double &zPB);
void penalty(unsigned int it, unsigned int nt, double a[3], double b[3], double c[3], double *d[3], double *e[3],
             double *f[3], double *p[3], double *q[3]);
void hybrid(int it, int nt, double a[3], double b[3], double c[3], double *d[3], double *e[3], double *f[3],
            double *p[3], double *q[3]);

extern "C" {

// One pair; pq holds the caller's values on entry (the reference leaves them untouched
// on its early return).
void zref_bf(const double *xA, const double *yA, const double *zA, const double *xB, const double *yB,
             const double *zB, double pq[6]) {
  double xa[3], ya[3], za[3], xb[3], yb[3], zb[3];
  for (int k = 0; k < 3; ++k) {
    xa[k] = xA[k]; ya[k] = yA[k]; za[k] = zA[k];
    xb[k] = xB[k]; yb[k] = yB[k]; zb[k] = zB[k];
  }
  bf(xa, ya, za, xb, yb, zb, pq[0], pq[1], pq[2], pq[3], pq[4], pq[5]);
}

void zref_penalty(uint32_t it, uint32_t nt, const double *a, const double *b, const double *c, double *d, double *e,
                  double *f, int64_t ld, double *p, double *q) {
  double A[3] = {a[0], a[1], a[2]}, B[3] = {b[0], b[1], b[2]}, Cc[3] = {c[0], c[1], c[2]};
  double *D[3] = {d, d + ld, d + 2 * ld}, *E[3] = {e, e + ld, e + 2 * ld}, *F[3] = {f, f + ld, f + 2 * ld};
  double *P[3] = {p, p + ld, p + 2 * ld}, *Q[3] = {q, q + ld, q + 2 * ld};
  penalty(it, nt, A, B, Cc, D, E, F, P, Q);
}

void zref_hybrid(int32_t it, int32_t nt, const double *a, const double *b, const double *c, double *d, double *e,
                 double *f, int64_t ld, double *p, double *q) {
  double A[3] = {a[0], a[1], a[2]}, B[3] = {b[0], b[1], b[2]}, Cc[3] = {c[0], c[1], c[2]};
  double *D[3] = {d, d + ld, d + 2 * ld}, *E[3] = {e, e + ld, e + 2 * ld}, *F[3] = {f, f + ld, f + 2 * ld};
  double *P[3] = {p, p + ld, p + 2 * ld}, *Q[3] = {q, q + ld, q + 2 * ld};
  hybrid(it, nt, A, B, Cc, D, E, F, P, Q);
}

}  // extern "C"
