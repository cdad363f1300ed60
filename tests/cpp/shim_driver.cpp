// Calls the C++ host layer (delta_b200.hpp) with the reference's driver signatures.
// Input (binary, little endian): int32 nA, nB; then xA,yA,zA (3*nA doubles each), xB,yB,zB;
// double epsA, epsB.  Output: one line per driver and contact, doubles in %a form.
#include <cstdio>
#include <vector>

#include "delta_b200.hpp"

namespace g = delta::contact::detection::gpu;

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  FILE *f = std::fopen(argv[1], "rb");
  if (!f) return 2;
  int nA = 0, nB = 0;
  if (std::fread(&nA, 4, 1, f) != 1 || std::fread(&nB, 4, 1, f) != 1) return 2;
  std::vector<double> a(9 * nA), b(9 * nB);
  double eps[2];
  if (std::fread(a.data(), 8, a.size(), f) != a.size() || std::fread(b.data(), 8, b.size(), f) != b.size() ||
      std::fread(eps, 8, 2, f) != 2)
    return 2;
  std::fclose(f);
  const double *xA = a.data(), *yA = xA + 3 * nA, *zA = yA + 3 * nA;
  const double *xB = b.data(), *yB = xB + 3 * nB, *zB = yB + 3 * nB;
  auto print = [](const char *name, const g::Contacts &c) {
    for (const auto &p : c)
      std::printf("%s %a %a %a %a %a %a %a %a %a %d %d %d\n", name, p.x[0], p.x[1], p.x[2], p.normal[0],
                  p.normal[1], p.normal[2], p.depth, p.P[0], p.Q[0], p.master, p.slave, (int)p.friction);
  };
  print("bf", g::bf(xA, yA, zA, nA, eps[0], true, 3, xB, yB, zB, nB, eps[1], true, 8));
  print("penalty", g::penalty(xA, yA, zA, nA, eps[0], true, 3, xB, yB, zB, nB, eps[1], true, 8));
  print("hybrid_batch", g::hybridWithPerBatchFallBack(xA, yA, zA, nA, eps[0], true, 3, xB, yB, zB, nB, eps[1],
                                                      true, 8));
  print("bf_cert", g::bfCertified(xA, yA, zA, nA, eps[0], true, 3, xB, yB, zB, nB, eps[1], true, 8));
  print("penalty_stat", g::penaltyStat(xA, yA, zA, nA, eps[0], true, 3, xB, yB, zB, nB, eps[1], true, 8));
  const auto st = g::lastStatistics();
  std::printf("hist");
  for (long long v : st.newtonIterations) std::printf(" %lld", v);
  std::printf("\n");
  return 0;
}
