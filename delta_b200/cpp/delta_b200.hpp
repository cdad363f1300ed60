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

// Per triangle pair, one GPU launch per call (the batched form is the C ABI's
// delta_pairs_run): bfSolver (bf.h:92-107), penaltySolver with `failed` (penalty.h:117-131)
// and with the Newton iteration count (penalty.h:137-152; the count is written when the
// iteration exits early, as the reference does -- its caller penaltyStat starts it at 0).
void bfSolver(const double *xA, const double *yA, const double *zA, const double *xB, const double *yB,
              const double *zB, double &xPA, double &yPA, double &zPA, double &xPB, double &yPB, double &zPB);
void penaltySolver(const double *xA, const double *yA, const double *zA, const double *xB, const double *yB,
                   const double *zB, double &xPA, double &yPA, double &zPA, double &xPB, double &yPB, double &zPB,
                   double MaxErrorOfPenaltyMethod, bool &failed);
void penaltySolver(const double *xA, const double *yA, const double *zA, const double *xB, const double *yB,
                   const double *zB, double &xPA, double &yPA, double &zPA, double &xPB, double &yPB, double &zPB,
                   double maxError, int &numberOfNewtonIterationsRequired);

}  // namespace gpu
}  // namespace detection

namespace forces {
namespace gpu {
// The constants of forces.cpp:11-21 (SPRING, DAMPER, FRICTION; SSPRING, SDAMPER,
// SFRICTIONGOLD for spheres), which the reference fixes at compile time; settable here.
struct Constants {
  double spring = 1E4, damper = 0.5, friction = 0.5;
  double sphereSpring = 2E5, sphereDamper = 0.5, sphereFriction = 1;
};
Constants &constants();
// getContactsForces (forces.h:143-167): force and torque on A from its contacts with B,
// added onto force[3] and torque[3].  The referential positions, inverse inertias,
// rotations and materials are accepted and, as in the reference's result, not used.
void getContactsForces(std::vector<contactpoint> &conpnt, double positionASpatial[3], double positionAReferential[3],
                       double angularA[3], double refAngularA[3], double linearA[3], double massA,
                       double inverseA[9], double rotationA[9], int materialA, double positionBSpatial[3],
                       double positionBReferential[3], double angularB[3], double refAngularB[3],
                       double linearB[3], double massB, double inverseB[9], double rotationB[9], int materialB,
                       double force[3], double torque[3], bool isSphere);
}  // namespace gpu
}  // namespace forces
}  // namespace contact

namespace dynamics {
namespace gpu {
// dynamics.h:29-86
void updateAngular(double *refAngular, double *rotation, double *inertia, double *inverse, double *torque,
                   double step);
void updateRotationMatrix(double *angular, double *refAngular, double *rotation, double step);
void updateVertices(double *x, double *y, double *z, double *refx, double *refy, double *refz, double *rotation,
                    double *position, double *refposition);
}  // namespace gpu
}  // namespace dynamics
}  // namespace delta

// ---- the zoltan/ front end ----------------------------------------------------------------
// The functions of zoltan/{bf,penalty,hybrid,dynamics,forces}.h with their argument lists
// (host arrays), run on the GPU through delta_zoltan_* (include/delta_b200.h).  They live in
// namespace zoltan_gpu.  Compiled inside the reference's build, define
// DELTA_B200_ZOLTAN_CONTACTPOINT to its header ("contact.h") to use its struct contactpoint;
// otherwise a struct with the same fields (zoltan/contact.h:32-42) is declared here.
// struct loba and the rank are accepted and not used: everything runs on one GPU.
#ifdef DELTA_B200_ZOLTAN_CONTACTPOINT
#include DELTA_B200_ZOLTAN_CONTACTPOINT
namespace zoltan_gpu {
using ::contactpoint;
}
#else
namespace zoltan_gpu {
struct contactpoint {
  int pid[2];
  int color[2];
  double point[3];
  double normal[3];
  double depth;
  double pp[3];
  double qq[3];
};
}  // namespace zoltan_gpu
#endif
struct loba;

namespace zoltan_gpu {
// zoltan/bf.h:61-64, penalty.h:47-50, hybrid.h:45-48
void bf(unsigned int it, unsigned int nt, double A[3], double B[3], double C[3], double *D[3], double *E[3],
        double *F[3], double *P[3], double *Q[3]);
void penalty(unsigned int it, unsigned int nt, double a[3], double b[3], double c[3], double *d[3], double *e[3],
             double *f[3], double *p[3], double *q[3]);
void hybrid(int it, int nt, double a[3], double b[3], double c[3], double *d[3], double *e[3], double *f[3],
            double *p[3], double *q[3]);

// material::iparam[SPRING][GRANULAR] and [DAMPER][GRANULAR] (zoltan/material.h), which
// zoltan/delta.cpp:69-70 sets to 1e2 and 1.
struct Granular {
  double spring = 1E2, damper = 1;
};
Granular &granular();

namespace dynamics {
// zoltan/dynamics.h:37-49
void integrate(double step, double lo[3], double hi[3], int nt, double *t[3][3], double *v[3]);
void euler(int nb, double *angular[6], double *linear[3], double *rotation[9], double *position[6], double step);
void update(struct loba *lb, int myrank, std::vector<contactpoint> conpnt[], int nt, int nb, double *t[6][3],
            int pid[], double *angular[6], double *linear[3], double *rotation[9], double *position[6],
            double *inertia[9], double *inverse[9], double mass[], double *force[3], double *torque[3],
            double step, double lo[3], double hi[3]);
}  // namespace dynamics

namespace forces {
// zoltan/forces.h:35-37; conpnt[i] is emptied, as the reference does (forces.cpp:146)
void force(struct loba *lb, int myrank, std::vector<contactpoint> conpnt[], int nb, double *position[6],
           double *angular[6], double *linear[3], double mass[], double *force[3], double *torque[3],
           double gravity[3], int parmat[]);
}  // namespace forces
}  // namespace zoltan_gpu
