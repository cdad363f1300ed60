// Calls the C++ host layer (delta_b200.hpp) with the reference's per-call signatures:
// bfSolver / penaltySolver (bf.h, penalty.h), getContactsForces (forces.h), updateAngular /
// updateRotationMatrix / updateVertices (dynamics.h), and the zoltan/ functions (bf,
// penalty, hybrid, dynamics::update/euler/integrate, forces::force).
//
// Usage: shim_calls <mode> <input file>; the input is little-endian doubles (counts are
// stored as doubles too), laid out per mode as read below.  Output: one value per line
// in %a form, in the order written below.
#include <cstdio>
#include <string>
#include <vector>

#include "delta_b200.hpp"

namespace det = delta::contact::detection::gpu;
namespace frc = delta::contact::forces::gpu;
namespace dyn = delta::dynamics::gpu;

static std::vector<double> g_in;
static size_t g_pos = 0;
static double next() { return g_in.at(g_pos++); }
static int next_int() { return (int)next(); }
static void out(double v) { std::printf("%a\n", v); }

static void mode_pairs() {
  const int n = next_int();
  const double max_err = next();
  for (int i = 0; i < n; ++i) {
    double a[9], b[9];
    for (double &v : a) v = next();
    for (double &v : b) v = next();
    const double xA[3] = {a[0], a[3], a[6]}, yA[3] = {a[1], a[4], a[7]}, zA[3] = {a[2], a[5], a[8]};
    const double xB[3] = {b[0], b[3], b[6]}, yB[3] = {b[1], b[4], b[7]}, zB[3] = {b[2], b[5], b[8]};
    double p[6];
    det::bfSolver(xA, yA, zA, xB, yB, zB, p[0], p[1], p[2], p[3], p[4], p[5]);
    for (double v : p) out(v);
    bool failed = true;
    det::penaltySolver(xA, yA, zA, xB, yB, zB, p[0], p[1], p[2], p[3], p[4], p[5], max_err, failed);
    for (double v : p) out(v);
    out(failed ? 1.0 : 0.0);
    int iters = 0;
    det::penaltySolver(xA, yA, zA, xB, yB, zB, p[0], p[1], p[2], p[3], p[4], p[5], max_err, iters);
    for (double v : p) out(v);
    out(iters);
  }
}

static void mode_forces() {
  const int n = next_int();
  const bool sphere = next_int() != 0;
  std::vector<delta::contact::contactpoint> c(n);
  for (int i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) c[i].x[k] = next();
    for (int k = 0; k < 3; ++k) c[i].normal[k] = next();
    c[i].depth = next();
    c[i].friction = next_int() != 0;
  }
  double posA[3], angA[3], linA[3], posB[3], angB[3], linB[3], F[3], T[3], none[9] = {};
  for (double &v : posA) v = next();
  for (double &v : angA) v = next();
  for (double &v : linA) v = next();
  const double mA = next();
  for (double &v : posB) v = next();
  for (double &v : angB) v = next();
  for (double &v : linB) v = next();
  const double mB = next();
  for (double &v : F) v = next();
  for (double &v : T) v = next();
  frc::getContactsForces(c, posA, none, angA, none, linA, mA, none, none, 0, posB, none, angB, none, linB, mB, none,
                         none, 0, F, T, sphere);
  for (double v : F) out(v);
  for (double v : T) out(v);
}

static void mode_dynamics() {
  double W[3], R[9], J[9], Ji[9], tq[3], ang[3], x, y, z, rx, ry, rz, pos[3], rpos[3];
  for (double &v : W) v = next();
  for (double &v : R) v = next();
  for (double &v : J) v = next();
  for (double &v : Ji) v = next();
  for (double &v : tq) v = next();
  const double step = next();
  rx = next(), ry = next(), rz = next();
  for (double &v : pos) v = next();
  for (double &v : rpos) v = next();
  dyn::updateAngular(W, R, J, Ji, tq, step);
  dyn::updateRotationMatrix(ang, W, R, step);
  dyn::updateVertices(&x, &y, &z, &rx, &ry, &rz, R, pos, rpos);
  for (double v : W) out(v);
  for (double v : ang) out(v);
  for (double v : R) out(v);
  out(x), out(y), out(z);
}

static void mode_znarrow() {
  const int n = next_int();
  double abc[3][3];
  for (auto &r : abc)
    for (double &v : r) v = next();
  std::vector<double> lst(9 * (size_t)n);
  for (double &v : lst) v = next();
  const int it = next_int(), nt = next_int();
  for (int method = 0; method < 3; ++method) {
    std::vector<double> pq(6 * (size_t)n, 7.0);
    double *D[3], *E[3], *F[3], *P[3], *Q[3];
    for (int k = 0; k < 3; ++k) {
      D[k] = lst.data() + (size_t)k * n;
      E[k] = lst.data() + (size_t)(3 + k) * n;
      F[k] = lst.data() + (size_t)(6 + k) * n;
      P[k] = pq.data() + (size_t)k * n;
      Q[k] = pq.data() + (size_t)(3 + k) * n;
    }
    if (method == 0) zoltan_gpu::bf(it, nt, abc[0], abc[1], abc[2], D, E, F, P, Q);
    else if (method == 1) zoltan_gpu::penalty(it, nt, abc[0], abc[1], abc[2], D, E, F, P, Q);
    else zoltan_gpu::hybrid(it, nt, abc[0], abc[1], abc[2], D, E, F, P, Q);
    for (double v : pq) out(v);
  }
}

static void mode_zsystem() {
  const int nb = next_int(), nt = next_int(), nc = next_int();
  const double step = next();
  double g[3];
  for (double &v : g) v = next();
  auto planes = [](int k, int n) {
    std::vector<double> v((size_t)k * n);
    for (double &x : v) x = next();
    return v;
  };
  std::vector<double> t = planes(18, nt), ang = planes(6, nb), lin = planes(3, nb), rot = planes(9, nb),
                      pos = planes(6, nb), J = planes(9, nb), Ji = planes(9, nb), mass = planes(1, nb),
                      F = planes(3, nb), T = planes(3, nb);
  std::vector<int> pid(nt);
  for (int &p : pid) p = next_int();
  std::vector<std::vector<zoltan_gpu::contactpoint>> con(nb);
  for (int c = 0; c < nc; ++c) {
    zoltan_gpu::contactpoint cp{};
    cp.pid[0] = next_int();
    cp.pid[1] = next_int();
    for (double &v : cp.point) v = next();
    for (double &v : cp.normal) v = next();
    cp.depth = next();
    con.at(cp.pid[0]).push_back(cp);
  }
  auto ptrs = [](std::vector<double> &v, int k, int n) {
    std::vector<double *> p(k);
    for (int j = 0; j < k; ++j) p[j] = v.data() + (size_t)j * n;
    return p;
  };
  auto pa = ptrs(ang, 6, nb), pl = ptrs(lin, 3, nb), pr = ptrs(rot, 9, nb), px = ptrs(pos, 6, nb),
       pj = ptrs(J, 9, nb), pi = ptrs(Ji, 9, nb), pf = ptrs(F, 3, nb), pt = ptrs(T, 3, nb);
  // forces::force, then dynamics::update, then euler, then integrate on the spatial vertices
  zoltan_gpu::forces::force(nullptr, 0, con.data(), nb, px.data(), pa.data(), pl.data(), mass.data(), pf.data(),
                            pt.data(), g, nullptr);
  for (double v : F) out(v);
  for (double v : T) out(v);
  double *tt[6][3];
  for (int w = 0; w < 6; ++w)
    for (int k = 0; k < 3; ++k) tt[w][k] = t.data() + (size_t)(3 * w + k) * nt;
  double lo[3] = {-1, -1, -1}, hi[3] = {1, 1, 1};
  zoltan_gpu::dynamics::update(nullptr, 0, con.data(), nt, nb, tt, pid.data(), pa.data(), pl.data(), pr.data(),
                               px.data(), pj.data(), pi.data(), mass.data(), pf.data(), pt.data(), step, lo, hi);
  for (auto *v : {&t, &ang, &lin, &rot, &pos, &F, &T})
    for (double x : *v) out(x);
  zoltan_gpu::dynamics::euler(nb, pa.data(), pl.data(), pr.data(), px.data(), step);
  for (auto *v : {&ang, &rot, &pos})
    for (double x : *v) out(x);
  std::vector<double> vel((size_t)3 * nt);
  for (size_t i = 0; i < vel.size(); ++i) vel[i] = t[i] - t[(size_t)9 * nt + i];  // any values
  double *tv[3][3], *pv[3];
  for (int w = 0; w < 3; ++w)
    for (int k = 0; k < 3; ++k) tv[w][k] = tt[w][k];
  for (int k = 0; k < 3; ++k) pv[k] = vel.data() + (size_t)k * nt;
  zoltan_gpu::dynamics::integrate(step, lo, hi, nt, tv, pv);
  for (size_t i = 0; i < (size_t)9 * nt; ++i) out(t[i]);
  for (double x : vel) out(x);
}

int main(int argc, char **argv) {
  if (argc < 3) return 2;
  FILE *f = std::fopen(argv[2], "rb");
  if (!f) return 2;
  double v;
  while (std::fread(&v, 8, 1, f) == 1) g_in.push_back(v);
  std::fclose(f);
  const std::string mode = argv[1];
  if (mode == "pairs") mode_pairs();
  else if (mode == "forces") mode_forces();
  else if (mode == "dynamics") mode_dynamics();
  else if (mode == "znarrow") mode_znarrow();
  else if (mode == "zsystem") mode_zsystem();
  else return 2;
  return 0;
}
