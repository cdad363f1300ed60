// ref_shim.cpp -- extern "C" entry points over the reference's own hot-path functions.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with the
// reference's sources (delta/contact/..., delta/dynamics/...) where they lie, into
// oracle/_ref/.  The result pins the C restatement (delta_oracle.c) and serves as the
// timed CPU baseline.  Nothing in the product path loads it.
#include <cstdint>
#include <cstring>
#include <vector>

#include "contact/contactpoint.h"
#include "contact/filter.h"
#include "contact/detection/point.h"
#include "contact/detection/sphere.h"
#include "contact/detection/bf.h"
#include "contact/detection/gjk.h"
#include "contact/detection/hybrid.h"
#include "contact/detection/penalty.h"
#include "contact/forces/forces.h"
#include "dynamics/dynamics.h"

#include <thread>

void expmap(iREAL, iREAL, iREAL, iREAL &, iREAL &, iREAL &, iREAL &, iREAL &, iREAL &, iREAL &, iREAL &,
            iREAL &);

namespace det = delta::contact::detection;

extern "C" {

// Same field order as dor_contact in delta_oracle.h.
struct ref_contact {
  double x[3], normal[3], depth, P[3], Q[3];
  int32_t friction;
  double eps_total;
  int32_t master, slave, penetration, tri_a, tri_b;
};

struct ref_stats {
  int64_t newton_hist[17];
  int64_t penalty_fails, batch_fails, batch_size;
  double batch_error;
};

void ref_bf_solver(const double *xA, const double *yA, const double *zA, const double *xB, const double *yB,
                   const double *zB, double pq[6]) {
  det::bfSolver(xA, yA, zA, xB, yB, zB, pq[0], pq[1], pq[2], pq[3], pq[4], pq[5]);
}

void ref_penalty_solver(const double *xA, const double *yA, const double *zA, const double *xB,
                        const double *yB, const double *zB, double max_error, double pq[6], int32_t *failed) {
  bool f = false;
  det::penaltySolver(xA, yA, zA, xB, yB, zB, pq[0], pq[1], pq[2], pq[3], pq[4], pq[5], max_error, f);
  *failed = f ? 1 : 0;
}

void ref_penalty_solver_iter(const double *xA, const double *yA, const double *zA, const double *xB,
                             const double *yB, const double *zB, double max_error, double pq[6],
                             int32_t *iterations) {
  int it = *iterations;
  det::penaltySolver(xA, yA, zA, xB, yB, zB, pq[0], pq[1], pq[2], pq[3], pq[4], pq[5], max_error, it);
  *iterations = it;
}

double ref_gjk(const double *a, int32_t na, const double *b, int32_t nb, double p[3], double q[3]) {
  return det::gjk(const_cast<double *>(a), na, const_cast<double *>(b), nb, p, q);
}

static inline double pq_dist(const double *pq) {
  return std::sqrt(((pq[3] - pq[0]) * (pq[3] - pq[0])) + ((pq[4] - pq[1]) * (pq[4] - pq[1])) +
                   ((pq[5] - pq[2]) * (pq[5] - pq[2])));
}

// Pair list: plane k = 3*vertex + coord, element i.  method: 0 bf, 1 penalty (4 it),
// 2 penalty (<=16 it), 3 gjk(a,3,b,3), 4 per-pair hybrid (penalty, bf when failed).
static void pairs_range(int32_t method, int64_t i0, int64_t i1, const double *a, const double *b, int64_t ld,
                        double max_error, double *p, double *q, double *dist, uint8_t *flags) {
  for (int64_t i = i0; i < i1; ++i) {
    double xA[3], yA[3], zA[3], xB[3], yB[3], zB[3], pq[6];
    for (int v = 0; v < 3; ++v) {
      xA[v] = a[(3 * v + 0) * ld + i];
      yA[v] = a[(3 * v + 1) * ld + i];
      zA[v] = a[(3 * v + 2) * ld + i];
      xB[v] = b[(3 * v + 0) * ld + i];
      yB[v] = b[(3 * v + 1) * ld + i];
      zB[v] = b[(3 * v + 2) * ld + i];
    }
    int32_t flag = 0;
    if (method == 0) {
      ref_bf_solver(xA, yA, zA, xB, yB, zB, pq);
    } else if (method == 1) {
      ref_penalty_solver(xA, yA, zA, xB, yB, zB, max_error, pq, &flag);
    } else if (method == 2) {
      ref_penalty_solver_iter(xA, yA, zA, xB, yB, zB, max_error, pq, &flag);
    } else if (method == 3) {
      double aa[9], bb[9];
      for (int v = 0; v < 3; ++v) {
        aa[3 * v] = xA[v]; aa[3 * v + 1] = yA[v]; aa[3 * v + 2] = zA[v];
        bb[3 * v] = xB[v]; bb[3 * v + 1] = yB[v]; bb[3 * v + 2] = zB[v];
      }
      ref_gjk(aa, 3, bb, 3, pq, pq + 3);
    } else {
      ref_penalty_solver(xA, yA, zA, xB, yB, zB, max_error, pq, &flag);
      if (flag) ref_bf_solver(xA, yA, zA, xB, yB, zB, pq);
    }
    for (int k = 0; k < 3; ++k) {
      p[k * ld + i] = pq[k];
      q[k * ld + i] = pq[3 + k];
    }
    dist[i] = pq_dist(pq);
    if (flags) flags[i] = (uint8_t)flag;
  }
}

// nthreads <= 0 uses every hardware thread; the pairs are split into equal static blocks.
void ref_pairs(int32_t method, int64_t n, const double *a, const double *b, int64_t ld, double max_error,
               double *p, double *q, double *dist, uint8_t *flags, int32_t nthreads) {
  int64_t nt = nthreads > 0 ? nthreads : (int64_t)std::thread::hardware_concurrency();
  if (nt < 1) nt = 1;
  if (nt > n) nt = n > 0 ? n : 1;
  std::vector<std::thread> pool;
  for (int64_t t = 1; t < nt; ++t)
    pool.emplace_back(pairs_range, method, n * t / nt, n * (t + 1) / nt, a, b, ld, max_error, p, q, dist, flags);
  pairs_range(method, 0, n / nt, a, b, ld, max_error, p, q, dist, flags);
  for (auto &th : pool) th.join();
}

// Particle-pair drivers.  driver: 0 bf, 1 penalty, 2 penaltyStat, 3 hybridWithPerBatchFallBack,
// 4 hybridWithPerTriangleFallBack, 5 hybridBatchStat, 6 hybridTriangleStat.
int64_t ref_detect(int32_t driver, const double *xA, const double *yA, const double *zA, int32_t nA, double epsA,
                   int32_t fricA, int32_t idA, const double *xB, const double *yB, const double *zB, int32_t nB,
                   double epsB, int32_t fricB, int32_t idB, ref_contact *out, int64_t cap, ref_stats *stats) {
  std::vector<delta::contact::contactpoint> r;
  if (stats) {
    det::cleanPenaltyStatistics();
    det::cleanHybridStatistics();
  }
  switch (driver) {
    case 0: r = det::bf(xA, yA, zA, nA, epsA, fricA, idA, xB, yB, zB, nB, epsB, fricB, idB); break;
    case 1: r = det::penalty(xA, yA, zA, nA, epsA, fricA, idA, xB, yB, zB, nB, epsB, fricB, idB); break;
    case 2: r = det::penaltyStat(xA, yA, zA, nA, epsA, fricA, idA, xB, yB, zB, nB, epsB, fricB, idB); break;
    case 3:
      r = det::hybridWithPerBatchFallBack(xA, yA, zA, nA, epsA, fricA, idA, xB, yB, zB, nB, epsB, fricB, idB);
      break;
    case 4:
      r = det::hybridWithPerTriangleFallBack(xA, yA, zA, nA, epsA, fricA, idA, xB, yB, zB, nB, epsB, fricB, idB);
      break;
    case 5: r = det::hybridBatchStat(xA, yA, zA, nA, epsA, fricA, idA, xB, yB, zB, nB, epsB, fricB, idB); break;
    case 6: r = det::hybridTriangleStat(xA, yA, zA, nA, epsA, fricA, idA, xB, yB, zB, nB, epsB, fricB, idB); break;
    default: return -1;
  }
  if (stats) {
    std::vector<int> h = det::getPenaltyIterationStatistics();
    for (int i = 0; i < 17 && i < (int)h.size(); ++i) stats->newton_hist[i] = h[i];
    stats->penalty_fails = det::getPenaltyFails();
    stats->batch_fails = det::getBatchFails();
    stats->batch_size = det::getBatchSize();
    stats->batch_error = det::getBatchError();
  }
  const int64_t n = (int64_t)r.size();
  for (int64_t i = 0; i < n && i < cap; ++i) {
    const auto &c = r[i];
    ref_contact &o = out[i];
    std::memcpy(o.x, c.x, sizeof o.x);
    std::memcpy(o.normal, c.normal, sizeof o.normal);
    o.depth = c.depth;
    std::memcpy(o.P, c.P, sizeof o.P);
    std::memcpy(o.Q, c.Q, sizeof o.Q);
    o.friction = c.friction ? 1 : 0;
    o.eps_total = c.epsilonTotal;
    o.master = c.master;
    o.slave = c.slave;
    o.penetration = c.penetration;
    o.tri_a = -1;
    o.tri_b = -1;
  }
  return n;
}

// getContactsForces (mesh path) over nc contacts given as ref_contact records; the
// spring, damper and friction constants are the ones compiled into forces.cpp.
void ref_contacts_forces(const ref_contact *cp, int64_t nc, double *posA, double *angA, double *linA, double massA,
                         double *posB, double *angB, double *linB, double massB, double force[3],
                         double torque[3]) {
  std::vector<delta::contact::contactpoint> v((size_t)nc);
  for (int64_t i = 0; i < nc; ++i) {
    auto &c = v[i];
    std::memcpy(c.x, cp[i].x, sizeof c.x);
    std::memcpy(c.normal, cp[i].normal, sizeof c.normal);
    c.depth = cp[i].depth;
    std::memcpy(c.P, cp[i].P, sizeof c.P);
    std::memcpy(c.Q, cp[i].Q, sizeof c.Q);
    c.friction = cp[i].friction != 0;
    c.epsilonTotal = cp[i].eps_total;
    c.master = cp[i].master;
    c.slave = cp[i].slave;
    c.penetration = cp[i].penetration;
  }
  double refA[3] = {0, 0, 0}, refB[3] = {0, 0, 0}, refAngA[3] = {0, 0, 0}, refAngB[3] = {0, 0, 0};
  double I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  double RA[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, RB[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  delta::contact::forces::getContactsForces(v, posA, refA, angA, refAngA, linA, massA, I, RA, 0, posB, refB, angB,
                                            refAngB, linB, massB, I, RB, 0, force, torque, false);
}

void ref_expmap(double o1, double o2, double o3, double L[9]) {
  expmap(o1, o2, o3, L[0], L[1], L[2], L[3], L[4], L[5], L[6], L[7], L[8]);
}

void ref_update_rotation(double ang[3], double ref_ang[3], double rot[9], double step) {
  delta::dynamics::updateRotationMatrix(ang, ref_ang, rot, step);
}

void ref_update_angular(double ref_ang[3], double rot[9], double inertia[9], double inverse[9], double torque[3],
                        double step) {
  delta::dynamics::updateAngular(ref_ang, rot, inertia, inverse, torque, step);
}

void ref_update_vertex(double *x, double *y, double *z, double *rx, double *ry, double *rz, double rot[9],
                       double pos[3], double ref_pos[3]) {
  delta::dynamics::updateVertices(x, y, z, rx, ry, rz, rot, pos, ref_pos);
}

static void to_ref(const delta::contact::contactpoint &c, ref_contact &o) {
  std::memcpy(o.x, c.x, sizeof o.x);
  std::memcpy(o.normal, c.normal, sizeof o.normal);
  o.depth = c.depth;
  std::memcpy(o.P, c.P, sizeof o.P);
  std::memcpy(o.Q, c.Q, sizeof o.Q);
  o.friction = c.friction ? 1 : 0;
  o.eps_total = c.epsilonTotal;
  o.master = c.master;
  o.slave = c.slave;
  o.penetration = c.penetration;
  o.tri_a = -1;
  o.tri_b = -1;
}

// point.cpp:11 pt(), sphere.cpp sphere / sphereWithBarrierAB / BA / isSphereOverlayInContact
double ref_pt(const double *TP1, const double *TP2, const double *TP3, const double *c, double *tq) {
  double a[3], b[3], d[3], p[3];
  std::memcpy(a, TP1, sizeof a);
  std::memcpy(b, TP2, sizeof b);
  std::memcpy(d, TP3, sizeof d);
  std::memcpy(p, c, sizeof p);
  return det::pt(a, b, d, p, tq);
}

int64_t ref_sphere(const double *cA, double dA, double epsA, int32_t fA, int32_t idA, const double *cB, double dB,
                   double epsB, int32_t fB, int32_t idB, ref_contact *out) {
  auto r = det::sphere(cA[0], cA[1], cA[2], dA, epsA, fA != 0, idA, cB[0], cB[1], cB[2], dB, epsB, fB != 0, idB);
  if (!r.empty() && out) to_ref(r[0], out[0]);
  return (int64_t)r.size();
}

int64_t ref_sphere_mesh(int32_t ba, const double *c, double d, double epsS, int32_t fS, int32_t idS, const double *x,
                        const double *y, const double *z, int32_t nT, double epsM, int32_t fM, int32_t idM,
                        ref_contact *out, int64_t cap) {
  std::vector<delta::contact::contactpoint> r =
      ba == 0 ? det::sphereWithBarrierAB(c[0], c[1], c[2], d, epsS, fS != 0, idS, x, y, z, nT, epsM, fM != 0, idM)
              : det::sphereWithBarrierBA(c[0], c[1], c[2], d, epsS, fS != 0, idS, x, y, z, nT, epsM, fM != 0, idM);
  for (int64_t i = 0; i < (int64_t)r.size() && i < cap; ++i) to_ref(r[i], out[i]);
  return (int64_t)r.size();
}

int32_t ref_sphere_overlay(const double *cA, double rA, const double *cB, double rB) {
  return det::isSphereOverlayInContact(cA[0], cA[1], cA[2], rA, cB[0], cB[1], cB[2], rB) ? 1 : 0;
}

// filterNewContacts / filterOldContacts on one contact list each (x as 3 planes of ld
// doubles).  The contacts carry their index in `master`, so the survivors name themselves:
// keep[i] = 1 for every contact the reference function keeps.  Returns the survivors.
static std::vector<delta::contact::contactpoint> as_contacts(int64_t n, const double *x, int64_t ld) {
  std::vector<delta::contact::contactpoint> v(n);
  for (int64_t i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) v[i].x[k] = x[k * ld + i];
    v[i].master = (int)i;
  }
  return v;
}

int64_t ref_filter_new(int64_t n, const double *x, int64_t ld, uint8_t *keep) {
  std::vector<delta::contact::contactpoint> v = as_contacts(n, x, ld);
  delta::contact::filterNewContacts(v);
  std::memset(keep, 0, (size_t)n);
  for (const auto &c : v) keep[c.master] = 1;
  return (int64_t)v.size();
}

int64_t ref_filter_old(int64_t ns, const double *xs, int64_t lds, int64_t nn, const double *xn, int64_t ldn,
                       uint8_t *keep) {
  std::vector<delta::contact::contactpoint> stored = as_contacts(ns, xs, lds), fresh = as_contacts(nn, xn, ldn);
  delta::contact::filterOldContacts(stored, fresh);
  std::memset(keep, 0, (size_t)nn);
  for (const auto &c : fresh) keep[c.master] = 1;
  return (int64_t)fresh.size();
}

}  // extern "C"
