// delta_b200.cpp -- the C++ host layer over the C ABI (see delta_b200.hpp).
#include "delta_b200.hpp"

#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>

#include "delta_b200.h"

namespace delta {
namespace contact {
namespace detection {
namespace gpu {

namespace {

std::mutex g_mutex;
delta_ctx *g_ctx = nullptr;
Statistics g_stats;

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
  template <class T> T *as() const { return static_cast<T *>(p); }
};

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
