// delta_b200.hpp -- C++ host layer with the reference's detection signatures.
//
// The functions below take the arguments of delta::contact::detection::{bf, penalty,
// penaltyStat, hybridWithPerBatchFallBack, hybridWithPerTriangleFallBack,
// hybridBatchStat, hybridTriangleStat, gjk} (delta/contact/detection/{bf,penalty,hybrid,gjk}.h)
// and return the same std::vector<contactpoint>; they run on the GPU through the C ABI
// (include/delta_b200.h).  They live in namespace delta::contact::detection::gpu so that a
// C++ host can switch a call site by qualifying it.  Compiled inside the reference's
// build, define DELTA_B200_REFERENCE_CONTACTPOINT to its header (e.g.
// "contact/contactpoint.h") to use the reference's struct; otherwise a struct with the
// same fields (contactpoint.h:42-103) is declared here.
#pragma once
#include <cstdint>
#include <utility>
#include <vector>

#ifdef DELTA_B200_REFERENCE_CONTACTPOINT
#include DELTA_B200_REFERENCE_CONTACTPOINT
#else
namespace delta {
namespace contact {
struct contactpoint {
  double x[3];
  double normal[3];
  double depth;
  double P[3];
  double Q[3];
  bool friction;
  double epsilonTotal;
  int master;
  int slave;
  int penetration;
};
}  // namespace contact
}  // namespace delta
#endif

namespace delta {
namespace contact {
namespace detection {
namespace gpu {

using Contacts = std::vector<contactpoint>;

// bf.h:65-81
Contacts bf(const double *xA, const double *yA, const double *zA, int nA, double epsA, bool frictionA, int particleA,
            const double *xB, const double *yB, const double *zB, int nB, double epsB, bool frictionB, int particleB);
// penalty.h:99-115, penalty.h:59-74
Contacts penalty(const double *xA, const double *yA, const double *zA, int nA, double epsA, bool frictionA,
                 int particleA, const double *xB, const double *yB, const double *zB, int nB, double epsB,
                 bool frictionB, int particleB);
Contacts penaltyStat(const double *xA, const double *yA, const double *zA, int nA, double epsA, bool frictionA,
                     int particleA, const double *xB, const double *yB, const double *zB, int nB, double epsB,
                     bool frictionB, int particleB);
// hybrid.h:76-160
Contacts hybridWithPerBatchFallBack(const double *xA, const double *yA, const double *zA, int nA, double epsA,
                                    bool frictionA, int particleA, const double *xB, const double *yB,
                                    const double *zB, int nB, double epsB, bool frictionB, int particleB);
Contacts hybridWithPerTriangleFallBack(const double *xA, const double *yA, const double *zA, int nA, double epsA,
                                       bool frictionA, int particleA, const double *xB, const double *yB,
                                       const double *zB, int nB, double epsB, bool frictionB, int particleB);
Contacts hybridBatchStat(const double *xA, const double *yA, const double *zA, int nA, double epsA, bool frictionA,
                         int particleA, const double *xB, const double *yB, const double *zB, int nB, double epsB,
                         bool frictionB, int particleB);
Contacts hybridTriangleStat(const double *xA, const double *yA, const double *zA, int nA, double epsA,
                            bool frictionA, int particleA, const double *xB, const double *yB, const double *zB,
                            int nB, double epsB, bool frictionB, int particleB);
// gjk.h:32-47 argument order; per triangle pair with bf()'s contact rule
Contacts gjk(int nA, double *xA, double *yA, double *zA, double epsA, bool frictionA, int particleA, int nB,
             double *xB, double *yB, double *zB, double epsB, bool frictionB, int particleB);
// bf()'s contact set computed by the certified FP32 driver (equal to bf() bit for bit)
Contacts bfCertified(const double *xA, const double *yA, const double *zA, int nA, double epsA, bool frictionA,
                     int particleA, const double *xB, const double *yB, const double *zB, int nB, double epsB,
                     bool frictionB, int particleB);

// Many pairs in one call: bodies in SoA-tri layout, candidate pairs (indices into bodies).
struct Body {
  const double *x, *y, *z;
  int nTriangles;
  double epsilon;
  bool friction;
  int particle;
};
// driver: a delta_driver value (DELTA_DRV_BF = 0, ...).  Result k holds pair k's contacts.
std::vector<Contacts> detect(int driver, const std::vector<Body> &bodies,
                             const std::vector<std::pair<int, int>> &pairs);

// Statistics of the last penaltyStat / hybrid*Stat call (penalty.cpp:29-48, hybrid.cpp:27-56).
struct Statistics {
  std::vector<long long> newtonIterations;  // 17 bins
  long long penaltyFails = 0, batchFails = 0, batchSize = 0;
  double batchError = 0;
};
Statistics lastStatistics();

}  // namespace gpu
}  // namespace detection
}  // namespace contact
}  // namespace delta
