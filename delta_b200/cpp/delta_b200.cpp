// delta_b200.cpp -- the C++ host layer over the C ABI (see delta_b200.hpp).
#include "delta_b200.hpp"

#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>

#include "delta_b200.h"

// Shared by every function of this layer: one context on device 0, created on first use,
// and calls serialised by one mutex.
namespace delta_b200_host {

std::mutex g_mutex;
delta_ctx *g_ctx = nullptr;

void check_cuda(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string("delta_b200: ") + what + ": " + cudaGetErrorString(e));
}

void check(delta_status s) {
  if (s != DELTA_OK) throw std::runtime_error(std::string("delta_b200: ") + delta_last_error());
}

delta_ctx *context() {
  if (!g_ctx) check(delta_create(&g_ctx, 0, nullptr));
  return g_ctx;
}

// A device allocation released at scope exit.
struct DeviceBuffer {
  void *p = nullptr;
  explicit DeviceBuffer(size_t bytes) { check_cuda(cudaMalloc(&p, bytes ? bytes : 1), "cudaMalloc"); }
  ~DeviceBuffer() { cudaFree(p); }
  DeviceBuffer(const DeviceBuffer &) = delete;
  DeviceBuffer &operator=(const DeviceBuffer &) = delete;
  template <class T> T *as() const { return static_cast<T *>(p); }
};

void upload(void *dst, const void *src, size_t bytes) {
  if (bytes) check_cuda(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice), "upload");
}
void download(void *dst, const void *src, size_t bytes) {
  if (bytes) check_cuda(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost), "download");
}

}  // namespace delta_b200_host

namespace delta {
namespace contact {
namespace detection {
namespace gpu {

using namespace delta_b200_host;

namespace {
Statistics g_stats;
}  // namespace

std::vector<Contacts> detect(int driver, const std::vector<Body> &bodies,
                             const std::vector<std::pair<int, int>> &pairs) {
  std::lock_guard<std::mutex> lock(g_mutex);
  delta_ctx *ctx = context();
  const int n = (int)bodies.size();
  std::vector<int64_t> off(n + 1, 0);
  for (int i = 0; i < n; ++i) off[i + 1] = off[i] + bodies[i].nTriangles;
  const int64_t nv = 3 * off[n];
  std::vector<double> hx(nv), hy(nv), hz(nv), heps(n);
  std::vector<uint8_t> hfr(n);
  std::vector<int32_t> hid(n), hpa(pairs.size()), hpb(pairs.size());
  for (int i = 0; i < n; ++i) {
    const int64_t c = 3 * (int64_t)bodies[i].nTriangles;
    std::memcpy(hx.data() + 3 * off[i], bodies[i].x, sizeof(double) * c);
    std::memcpy(hy.data() + 3 * off[i], bodies[i].y, sizeof(double) * c);
    std::memcpy(hz.data() + 3 * off[i], bodies[i].z, sizeof(double) * c);
    heps[i] = bodies[i].epsilon;
    hfr[i] = bodies[i].friction ? 1 : 0;
    hid[i] = bodies[i].particle;
  }
  int64_t cap = 0;
  for (size_t k = 0; k < pairs.size(); ++k) {
    hpa[k] = pairs[k].first;
    hpb[k] = pairs[k].second;
    cap += (int64_t)bodies.at(pairs[k].first).nTriangles * bodies.at(pairs[k].second).nTriangles;
  }
  std::vector<Contacts> result(pairs.size());
  if (pairs.empty()) return result;
  DeviceBuffer dx(8 * nv), dy(8 * nv), dz(8 * nv), doff(8 * (n + 1)), deps(8 * n), dfr(n), did(4 * n),
      dpa(4 * pairs.size()), dpb(4 * pairs.size());
  check_cuda(cudaMemcpy(dx.p, hx.data(), 8 * nv, cudaMemcpyHostToDevice), "upload");
  check_cuda(cudaMemcpy(dy.p, hy.data(), 8 * nv, cudaMemcpyHostToDevice), "upload");
  check_cuda(cudaMemcpy(dz.p, hz.data(), 8 * nv, cudaMemcpyHostToDevice), "upload");
  check_cuda(cudaMemcpy(doff.p, off.data(), 8 * (n + 1), cudaMemcpyHostToDevice), "upload");
  check_cuda(cudaMemcpy(deps.p, heps.data(), 8 * n, cudaMemcpyHostToDevice), "upload");
  check_cuda(cudaMemcpy(dfr.p, hfr.data(), n, cudaMemcpyHostToDevice), "upload");
  check_cuda(cudaMemcpy(did.p, hid.data(), 4 * n, cudaMemcpyHostToDevice), "upload");
  check_cuda(cudaMemcpy(dpa.p, hpa.data(), 4 * pairs.size(), cudaMemcpyHostToDevice), "upload");
  check_cuda(cudaMemcpy(dpb.p, hpb.data(), 4 * pairs.size(), cudaMemcpyHostToDevice), "upload");
  delta_meshes m{n, doff.as<int64_t>(), dx.as<double>(), dy.as<double>(), dz.as<double>(), deps.as<double>(),
                 dfr.as<uint8_t>(), did.as<int32_t>()};
  // at most one contact per triangle pair; start smaller and grow on DELTA_ERR_CAPACITY
  int64_t c = cap < 4096 ? (cap > 0 ? cap : 1) : 4096;
  for (;;) {
    DeviceBuffer dd(8 * 14 * c), di(4 * 5 * c), df(c);
    double *d = dd.as<double>();
    int32_t *ip = di.as<int32_t>();
    delta_contacts out{c, d, d + 3 * c, d + 6 * c, d + 9 * c, d + 12 * c, d + 13 * c,
                       ip, ip + c, ip + 2 * c, ip + 3 * c, ip + 4 * c, df.as<uint8_t>()};
    int64_t nc = 0;
    delta_stats st;
    const delta_status s = delta_detect(ctx, driver, DELTA_F64, &m, dpa.as<int32_t>(), dpb.as<int32_t>(),
                                        (int64_t)pairs.size(), &out, &nc, &st);
    if (s == DELTA_ERR_CAPACITY) {
      c = nc;
      continue;
    }
    check(s);
    g_stats.newtonIterations.assign(st.newton_hist, st.newton_hist + 17);
    g_stats.penaltyFails = st.penalty_fails;
    g_stats.batchFails = st.batch_fails;
    g_stats.batchSize = st.batch_size;
    g_stats.batchError = st.batch_error;
    std::vector<double> h(14 * (size_t)nc);
    std::vector<int32_t> hi(5 * (size_t)nc);
    std::vector<uint8_t> hf((size_t)nc);
    for (int plane = 0; plane < 14; ++plane)
      check_cuda(cudaMemcpy(h.data() + plane * nc, d + plane * c, 8 * nc, cudaMemcpyDeviceToHost), "download");
    for (int plane = 0; plane < 5; ++plane)
      check_cuda(cudaMemcpy(hi.data() + plane * nc, ip + plane * c, 4 * nc, cudaMemcpyDeviceToHost), "download");
    check_cuda(cudaMemcpy(hf.data(), df.p, nc, cudaMemcpyDeviceToHost), "download");
    // contacts are ordered by pair, so they split into consecutive runs
    size_t k = 0;
    for (int64_t j = 0; j < nc; ++j) {
      const int32_t master = hi[j], slave = hi[nc + j];
      while (k < pairs.size() && !(hid[pairs[k].first] == master && hid[pairs[k].second] == slave)) ++k;
      if (k == pairs.size()) throw std::runtime_error("delta_b200: contact of an unknown pair");
      contactpoint cp{};
      for (int a = 0; a < 3; ++a) {
        cp.x[a] = h[a * nc + j];
        cp.normal[a] = h[(3 + a) * nc + j];
        cp.P[a] = h[(6 + a) * nc + j];
        cp.Q[a] = h[(9 + a) * nc + j];
      }
      cp.depth = h[12 * nc + j];
      cp.epsilonTotal = h[13 * nc + j];
      cp.friction = hf[j] != 0;
      cp.master = master;
      cp.slave = slave;
      cp.penetration = hi[4 * nc + j];
      result[k].push_back(cp);
    }
    return result;
  }
}

static Contacts one_pair(int driver, const double *xA, const double *yA, const double *zA, int nA, double epsA,
                         bool fA, int idA, const double *xB, const double *yB, const double *zB, int nB,
                         double epsB, bool fB, int idB) {
  std::vector<Body> bodies{{xA, yA, zA, nA, epsA, fA, idA}, {xB, yB, zB, nB, epsB, fB, idB}};
  return detect(driver, bodies, {{0, 1}})[0];
}

#define DELTA_B200_DRIVER(name, drv)                                                                              \
  Contacts name(const double *xA, const double *yA, const double *zA, int nA, double epsA, bool fA, int idA,     \
                const double *xB, const double *yB, const double *zB, int nB, double epsB, bool fB, int idB) {   \
    return one_pair(drv, xA, yA, zA, nA, epsA, fA, idA, xB, yB, zB, nB, epsB, fB, idB);                          \
  }
DELTA_B200_DRIVER(bf, DELTA_DRV_BF)
DELTA_B200_DRIVER(penalty, DELTA_DRV_PENALTY)
DELTA_B200_DRIVER(penaltyStat, DELTA_DRV_PENALTY_STAT)
DELTA_B200_DRIVER(hybridWithPerBatchFallBack, DELTA_DRV_HYBRID_BATCH)
DELTA_B200_DRIVER(hybridWithPerTriangleFallBack, DELTA_DRV_HYBRID_TRIANGLE)
DELTA_B200_DRIVER(hybridBatchStat, DELTA_DRV_HYBRID_BATCH_STAT)
DELTA_B200_DRIVER(hybridTriangleStat, DELTA_DRV_HYBRID_TRI_STAT)
DELTA_B200_DRIVER(bfCertified, DELTA_DRV_BF_CERT)
#undef DELTA_B200_DRIVER

Contacts gjk(int nA, double *xA, double *yA, double *zA, double epsA, bool fA, int idA, int nB, double *xB,
             double *yB, double *zB, double epsB, bool fB, int idB) {
  return one_pair(DELTA_DRV_GJK, xA, yA, zA, nA, epsA, fA, idA, xB, yB, zB, nB, epsB, fB, idB);
}

Statistics lastStatistics() {
  std::lock_guard<std::mutex> lock(g_mutex);
  return g_stats;
}

}  // namespace gpu
}  // namespace detection
}  // namespace contact
}  // namespace delta

// ---- per-pair solvers -----------------------------------------------------------------------
namespace delta {
using namespace delta_b200_host;
namespace contact {
namespace detection {
namespace gpu {

// One triangle pair through the pair-list entry point; returns the flag byte.
static int one_triangle_pair(int method, const double *xA, const double *yA, const double *zA, const double *xB,
                             const double *yB, const double *zB, double max_error, double pq[6]) {
  std::lock_guard<std::mutex> lock(g_mutex);
  double a[9], b[9], p[3], q[3], d;
  uint8_t flag = 0;
  for (int v = 0; v < 3; ++v) {
    a[3 * v] = xA[v], a[3 * v + 1] = yA[v], a[3 * v + 2] = zA[v];
    b[3 * v] = xB[v], b[3 * v + 1] = yB[v], b[3 * v + 2] = zB[v];
  }
  check(delta_pairs_run_host(context(), method, DELTA_F64, 1, a, b, 1, max_error, p, q, &d, &flag));
  for (int k = 0; k < 3; ++k) pq[k] = p[k], pq[3 + k] = q[k];
  return flag;
}

void bfSolver(const double *xA, const double *yA, const double *zA, const double *xB, const double *yB,
              const double *zB, double &xPA, double &yPA, double &zPA, double &xPB, double &yPB, double &zPB) {
  double pq[6];
  one_triangle_pair(DELTA_BF, xA, yA, zA, xB, yB, zB, 0.0, pq);
  xPA = pq[0], yPA = pq[1], zPA = pq[2], xPB = pq[3], yPB = pq[4], zPB = pq[5];
}

void penaltySolver(const double *xA, const double *yA, const double *zA, const double *xB, const double *yB,
                   const double *zB, double &xPA, double &yPA, double &zPA, double &xPB, double &yPB, double &zPB,
                   double MaxErrorOfPenaltyMethod, bool &failed) {
  double pq[6];
  failed = one_triangle_pair(DELTA_PENALTY, xA, yA, zA, xB, yB, zB, MaxErrorOfPenaltyMethod, pq) != 0;
  xPA = pq[0], yPA = pq[1], zPA = pq[2], xPB = pq[3], yPB = pq[4], zPB = pq[5];
}

void penaltySolver(const double *xA, const double *yA, const double *zA, const double *xB, const double *yB,
                   const double *zB, double &xPA, double &yPA, double &zPA, double &xPB, double &yPB, double &zPB,
                   double maxError, int &numberOfNewtonIterationsRequired) {
  double pq[6];
  const int it = one_triangle_pair(DELTA_PENALTY_ITER, xA, yA, zA, xB, yB, zB, maxError, pq);
  if (it != 0) numberOfNewtonIterationsRequired = it;
  xPA = pq[0], yPA = pq[1], zPA = pq[2], xPB = pq[3], yPB = pq[4], zPB = pq[5];
}

}  // namespace gpu
}  // namespace detection

// ---- getContactsForces ---------------------------------------------------------------------
namespace forces {
namespace gpu {

Constants &constants() {
  static Constants c;
  return c;
}

void getContactsForces(std::vector<contactpoint> &conpnt, double positionASpatial[3], double *, double angularA[3],
                       double *, double linearA[3], double massA, double *, double *, int,
                       double positionBSpatial[3], double *, double angularB[3], double *, double linearB[3],
                       double massB, double *, double *, int, double force[3], double torque[3], bool isSphere) {
  const int64_t n = (int64_t)conpnt.size();
  if (n == 0) return;
  std::lock_guard<std::mutex> lock(g_mutex);
  delta_ctx *ctx = context();
  std::vector<double> h(7 * (size_t)n);
  std::vector<uint8_t> fr((size_t)n);
  for (int64_t c = 0; c < n; ++c) {
    for (int k = 0; k < 3; ++k) {
      h[k * n + c] = conpnt[c].x[k];
      h[(3 + k) * n + c] = conpnt[c].normal[k];
    }
    h[6 * n + c] = conpnt[c].depth;
    fr[c] = conpnt[c].friction ? 1 : 0;
  }
  double kin[26];  // pos, ang, lin of A; mass A; pos, ang, lin of B; mass B; force; torque
  for (int k = 0; k < 3; ++k) {
    kin[k] = positionASpatial[k], kin[3 + k] = angularA[k], kin[6 + k] = linearA[k];
    kin[10 + k] = positionBSpatial[k], kin[13 + k] = angularB[k], kin[16 + k] = linearB[k];
    kin[20 + k] = force[k], kin[23 + k] = torque[k];
  }
  kin[9] = massA, kin[19] = massB;
  const int64_t off[2] = {0, n};
  DeviceBuffer dh(8 * h.size()), dfr((size_t)n), dkin(sizeof kin), doff(sizeof off);
  upload(dh.p, h.data(), 8 * h.size());
  upload(dfr.p, fr.data(), (size_t)n);
  upload(dkin.p, kin, sizeof kin);
  upload(doff.p, off, sizeof off);
  double *d = dh.as<double>(), *k = dkin.as<double>();
  delta_contacts cs{};
  cs.capacity = n;
  cs.x = d;
  cs.normal = d + 3 * n;
  cs.depth = d + 6 * n;
  cs.friction = dfr.as<uint8_t>();
  const Constants &C = constants();
  delta_step_params prm{};
  prm.spring = isSphere ? C.sphereSpring : C.spring;
  prm.damper = isSphere ? C.sphereDamper : C.damper;
  prm.friction = isSphere ? C.sphereFriction : C.friction;
  check(delta_contact_forces(ctx, 1, doff.as<int64_t>(), &cs, k, k + 3, k + 6, k + 9, k + 10, k + 13, k + 16, k + 19,
                             &prm, k + 20, k + 23));
  download(kin, dkin.p, sizeof kin);
  for (int j = 0; j < 3; ++j) force[j] = kin[20 + j], torque[j] = kin[23 + j];
}

}  // namespace gpu
}  // namespace forces
}  // namespace contact

// ---- dynamics --------------------------------------------------------------------------------
namespace dynamics {
namespace gpu {

void updateAngular(double *refAngular, double *rotation, double *inertia, double *inverse, double *torque,
                   double step) {
  std::lock_guard<std::mutex> lock(g_mutex);
  double h[33];
  std::memcpy(h, refAngular, 24);
  std::memcpy(h + 3, rotation, 72);
  std::memcpy(h + 12, inertia, 72);
  std::memcpy(h + 21, inverse, 72);
  std::memcpy(h + 30, torque, 24);
  DeviceBuffer d(sizeof h);
  upload(d.p, h, sizeof h);
  double *p = d.as<double>();
  check(delta_update_angular(context(), 1, p, p + 3, p + 12, p + 21, p + 30, step));
  download(refAngular, p, 24);
}

void updateRotationMatrix(double *angular, double *refAngular, double *rotation, double step) {
  std::lock_guard<std::mutex> lock(g_mutex);
  double h[15];
  std::memcpy(h, angular, 24);
  std::memcpy(h + 3, refAngular, 24);
  std::memcpy(h + 6, rotation, 72);
  DeviceBuffer d(sizeof h);
  upload(d.p, h, sizeof h);
  double *p = d.as<double>();
  check(delta_update_rotation(context(), 1, p, p + 3, p + 6, step));
  download(h, p, sizeof h);
  std::memcpy(angular, h, 24);
  std::memcpy(rotation, h + 6, 72);
}

void updateVertices(double *x, double *y, double *z, double *refx, double *refy, double *refz, double *rotation,
                    double *position, double *refposition) {
  std::lock_guard<std::mutex> lock(g_mutex);
  double h[21] = {0, 0, 0, *refx, *refy, *refz};
  std::memcpy(h + 6, rotation, 72);
  std::memcpy(h + 15, position, 24);
  std::memcpy(h + 18, refposition, 24);
  DeviceBuffer d(sizeof h);
  upload(d.p, h, sizeof h);
  double *p = d.as<double>();
  check(delta_update_vertices(context(), 1, nullptr, 1, p, p + 1, p + 2, p + 3, p + 4, p + 5, p + 6, p + 15,
                              p + 18));
  download(h, p, 24);
  *x = h[0], *y = h[1], *z = h[2];
}

}  // namespace gpu
}  // namespace dynamics
}  // namespace delta

// ---- the zoltan/ front end ----------------------------------------------------------------------
namespace zoltan_gpu {

using namespace delta_b200_host;

Granular &granular() {
  static Granular g;
  return g;
}

namespace {

// Per-coordinate host arrays of n doubles copied into one device block of k planes.
struct Planes {
  DeviceBuffer buf;
  int64_t n;
  int k;
  Planes(double *const *h, int k_, int64_t n_) : buf(8 * (size_t)k_ * (size_t)(n_ > 0 ? n_ : 1)), n(n_), k(k_) {
    for (int j = 0; j < k; ++j) upload(plane(j), h[j], 8 * (size_t)n);
  }
  double *plane(int j) const { return buf.as<double>() + (int64_t)j * (n > 0 ? n : 1); }
  void back(double *const *h) const {
    for (int j = 0; j < k; ++j) download(h[j], plane(j), 8 * (size_t)n);
  }
};

void narrow(int method, int64_t it, int64_t nt, double a[3], double b[3], double c[3], double *d[3], double *e[3],
            double *f[3], double *p[3], double *q[3]) {
  if (nt <= 0) return;
  std::lock_guard<std::mutex> lock(g_mutex);
  Planes D(d, 3, nt), E(e, 3, nt), F(f, 3, nt), P(p, 3, nt), Q(q, 3, nt);
  const double *dd[3] = {D.plane(0), D.plane(1), D.plane(2)}, *de[3] = {E.plane(0), E.plane(1), E.plane(2)},
               *df[3] = {F.plane(0), F.plane(1), F.plane(2)};
  double *dp[3] = {P.plane(0), P.plane(1), P.plane(2)}, *dq[3] = {Q.plane(0), Q.plane(1), Q.plane(2)};
  delta_ctx *ctx = context();
  if (method == 0) check(delta_zoltan_bf(ctx, (uint32_t)it, (uint32_t)nt, a, b, c, dd, de, df, dp, dq));
  else if (method == 1) check(delta_zoltan_penalty(ctx, (uint32_t)it, (uint32_t)nt, a, b, c, dd, de, df, dp, dq));
  else check(delta_zoltan_hybrid(ctx, (int32_t)it, (int32_t)nt, a, b, c, dd, de, df, dp, dq));
  check(delta_synchronize(ctx));
  P.back(p);
  Q.back(q);
}

}  // namespace

void bf(unsigned int it, unsigned int nt, double A[3], double B[3], double C[3], double *D[3], double *E[3],
        double *F[3], double *P[3], double *Q[3]) {
  narrow(0, it, nt, A, B, C, D, E, F, P, Q);
}
void penalty(unsigned int it, unsigned int nt, double a[3], double b[3], double c[3], double *d[3], double *e[3],
             double *f[3], double *p[3], double *q[3]) {
  narrow(1, it, nt, a, b, c, d, e, f, p, q);
}
void hybrid(int it, int nt, double a[3], double b[3], double c[3], double *d[3], double *e[3], double *f[3],
            double *p[3], double *q[3]) {
  if (it < 0) return;  // the reference's unsigned batch counter starts past every batch
  narrow(2, it, nt, a, b, c, d, e, f, p, q);
}

namespace dynamics {

void integrate(double step, double lo[3], double hi[3], int nt, double *t[3][3], double *v[3]) {
  if (nt <= 0) return;
  std::lock_guard<std::mutex> lock(g_mutex);
  double *tf[9];
  for (int w = 0; w < 3; ++w)
    for (int k = 0; k < 3; ++k) tf[3 * w + k] = t[w][k];
  Planes T(tf, 9, nt), V(v, 3, nt);
  double *dt[3][3], *dv[3] = {V.plane(0), V.plane(1), V.plane(2)};
  for (int w = 0; w < 3; ++w)
    for (int k = 0; k < 3; ++k) dt[w][k] = T.plane(3 * w + k);
  check(delta_zoltan_integrate(context(), step, lo, hi, nt, dt, dv));
  check(delta_synchronize(context()));
  T.back(tf);
  V.back(v);
}

void euler(int nb, double *angular[6], double *linear[3], double *rotation[9], double *position[6], double step) {
  if (nb <= 0) return;
  std::lock_guard<std::mutex> lock(g_mutex);
  Planes A(angular, 6, nb), L(linear, 3, nb), R(rotation, 9, nb), X(position, 6, nb);
  double *da[6], *dl[3], *dr[9], *dx[6];
  for (int k = 0; k < 6; ++k) da[k] = A.plane(k), dx[k] = X.plane(k);
  for (int k = 0; k < 3; ++k) dl[k] = L.plane(k);
  for (int k = 0; k < 9; ++k) dr[k] = R.plane(k);
  check(delta_zoltan_euler(context(), nb, da, dl, dr, dx, step));
  check(delta_synchronize(context()));
  A.back(angular);
  R.back(rotation);
  X.back(position);
}

void update(struct loba *, int, std::vector<contactpoint> *, int nt, int nb, double *t[6][3], int pid[],
            double *angular[6], double *linear[3], double *rotation[9], double *position[6], double *inertia[9],
            double *inverse[9], double mass[], double *force[3], double *torque[3], double step, double *,
            double *) {
  if (nb <= 0 && nt <= 0) return;
  std::lock_guard<std::mutex> lock(g_mutex);
  double *tf[18];
  for (int w = 0; w < 6; ++w)
    for (int k = 0; k < 3; ++k) tf[3 * w + k] = t[w][k];
  Planes T(tf, 18, nt), A(angular, 6, nb), L(linear, 3, nb), R(rotation, 9, nb), X(position, 6, nb),
      J(inertia, 9, nb), I(inverse, 9, nb), M(&mass, 1, nb), Fo(force, 3, nb), To(torque, 3, nb);
  DeviceBuffer dpid(4 * (size_t)(nt > 0 ? nt : 1));
  upload(dpid.p, pid, 4 * (size_t)(nt > 0 ? nt : 0));
  double *dt[6][3], *da[6], *dl[3], *dr[9], *dx[6], *dfo[3], *dto[3];
  const double *dj[9], *di[9];
  for (int w = 0; w < 6; ++w)
    for (int k = 0; k < 3; ++k) dt[w][k] = T.plane(3 * w + k);
  for (int k = 0; k < 6; ++k) da[k] = A.plane(k), dx[k] = X.plane(k);
  for (int k = 0; k < 3; ++k) dl[k] = L.plane(k), dfo[k] = Fo.plane(k), dto[k] = To.plane(k);
  for (int k = 0; k < 9; ++k) dr[k] = R.plane(k), dj[k] = J.plane(k), di[k] = I.plane(k);
  check(delta_zoltan_update(context(), nt, nb, dt, dpid.as<int32_t>(), da, dl, dr, dx, dj, di, M.plane(0), dfo, dto,
                            step));
  check(delta_synchronize(context()));
  T.back(tf);
  A.back(angular);
  L.back(linear);
  R.back(rotation);
  X.back(position);
  Fo.back(force);
  To.back(torque);
}

}  // namespace dynamics

namespace forces {

void force(struct loba *, int, std::vector<contactpoint> conpnt[], int nb, double *position[6], double *angular[6],
           double *linear[3], double mass[], double *force[3], double *torque[3], double gravity[3], int *) {
  if (nb <= 0) return;
  std::lock_guard<std::mutex> lock(g_mutex);
  std::vector<int64_t> off(nb + 1, 0);
  for (int i = 0; i < nb; ++i) off[i + 1] = off[i] + (int64_t)conpnt[i].size();
  const int64_t nc = off[nb];
  std::vector<double> pts(3 * (size_t)nc), nrm(3 * (size_t)nc), dep((size_t)nc);
  std::vector<int32_t> sl((size_t)nc);
  for (int i = 0; i < nb; ++i)
    for (size_t k = 0; k < conpnt[i].size(); ++k) {
      const int64_t c = off[i] + (int64_t)k;
      for (int j = 0; j < 3; ++j) {
        pts[j * nc + c] = conpnt[i][k].point[j];
        nrm[j * nc + c] = conpnt[i][k].normal[j];
      }
      dep[c] = conpnt[i][k].depth;
      sl[c] = conpnt[i][k].pid[1];
    }
  Planes X(position, 6, nb), A(angular, 6, nb), L(linear, 3, nb), M(&mass, 1, nb), Fo(force, 3, nb),
      To(torque, 3, nb);
  DeviceBuffer doff(8 * (size_t)(nb + 1)), dsl(4 * (size_t)(nc > 0 ? nc : 1)), dp(8 * pts.size() + 8),
      dn(8 * nrm.size() + 8), dd(8 * dep.size() + 8);
  upload(doff.p, off.data(), 8 * (size_t)(nb + 1));
  upload(dsl.p, sl.data(), 4 * (size_t)nc);
  upload(dp.p, pts.data(), 8 * pts.size());
  upload(dn.p, nrm.data(), 8 * nrm.size());
  upload(dd.p, dep.data(), 8 * dep.size());
  const double *dpt[3], *dnr[3], *dx[6], *da[6], *dl[3];
  double *dfo[3], *dto[3];
  for (int k = 0; k < 3; ++k) {
    dpt[k] = dp.as<double>() + k * nc;
    dnr[k] = dn.as<double>() + k * nc;
    dl[k] = L.plane(k), dfo[k] = Fo.plane(k), dto[k] = To.plane(k);
  }
  for (int k = 0; k < 6; ++k) dx[k] = X.plane(k), da[k] = A.plane(k);
  const Granular &g = granular();
  check(delta_zoltan_force(context(), nb, doff.as<int64_t>(), dsl.as<int32_t>(), nc, dpt, dnr, dd.as<double>(), dx,
                           da, dl, M.plane(0), dfo, dto, gravity, g.spring, g.damper));
  check(delta_synchronize(context()));
  Fo.back(force);
  To.back(torque);
  for (int i = 0; i < nb; ++i) std::vector<contactpoint>().swap(conpnt[i]);
}

}  // namespace forces
}  // namespace zoltan_gpu
