/*
 * delta_oracle.h -- CPU restatement (FP64) of the reference's per-timestep contact
 * pipeline for triangulated particles.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: tests/, the smoke check
 * and the CPU-baseline leg of bench.py load it.  The product path (delta_b200) never
 * links, loads or calls it.
 *
 * Every function cites the reference file:line whose arithmetic it follows.  The
 * library is compiled with -ffp-contract=off so that each a*b+c stays two rounded
 * operations, as in the reference compiled without FMA contraction.
 *
 * Layouts
 *   pair list  : a[9*ld], b[9*ld]; plane k = 3*vertex + coord, element i = pair i
 *                (the ispc_bf / ispc_pen pair-list shape, bf.ispc:3, penalty.ispc:154).
 *   SoA-tri    : x[3*nT], y[3*nT], z[3*nT]; triangle t owns entries 3t..3t+2
 *                (ParticleRecord _xCoordinates, bf.cpp:47-148).
 */
#ifndef DELTA_ORACLE_H
#define DELTA_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* struct contactpoint, contactpoint.h:42-103 */
typedef struct {
  double x[3];
  double normal[3];
  double depth;
  double P[3];
  double Q[3];
  int32_t friction;
  double eps_total;
  int32_t master;
  int32_t slave;
  int32_t penetration;
  int32_t tri_a;  /* triangle index in A (bookkeeping added here; not in the reference) */
  int32_t tri_b;  /* triangle index in B */
} dor_contact;

enum { DOR_BF = 0, DOR_PENALTY = 1, DOR_PENALTY_ITER = 2, DOR_GJK = 3, DOR_HYBRID_PAIR = 4 };

enum {
  DOR_DRV_BF = 0,               /* bf()                          bf.cpp:47-148          */
  DOR_DRV_PENALTY = 1,          /* penalty()                     penalty.cpp:133-275    */
  DOR_DRV_PENALTY_STAT = 2,     /* penaltyStat()                 penalty.cpp:50-110     */
  DOR_DRV_HYBRID_BATCH = 3,     /* hybridWithPerBatchFallBack    hybrid.cpp:357-487     */
  DOR_DRV_HYBRID_TRIANGLE = 4,  /* hybridWithPerTriangleFallBack hybrid.cpp:78-200      */
  DOR_DRV_HYBRID_BATCH_STAT = 5,/* hybridBatchStat               hybrid.cpp:489-628     */
  DOR_DRV_HYBRID_TRI_STAT = 6,  /* hybridTriangleStat            hybrid.cpp:202-336     */
  DOR_DRV_GJK = 7               /* gjk(a,3,b,3) per triangle pair, bf() contact rule    */
};

/* statistics kept by the stat drivers (penalty.cpp:29-48, hybrid.cpp:27-56) */
typedef struct {
  int64_t newton_hist[17];
  int64_t penalty_fails;
  int64_t batch_fails;
  int64_t batch_size;
  double batch_error;
} dor_stats;

/* ---- per triangle pair ------------------------------------------------------ */
void dor_bf_solver(const double *xA, const double *yA, const double *zA,
                   const double *xB, const double *yB, const double *zB, double pq[6]);
void dor_penalty_solver(const double *xA, const double *yA, const double *zA,
                        const double *xB, const double *yB, const double *zB,
                        double max_error, double pq[6], int32_t *failed);
void dor_penalty_solver_iter(const double *xA, const double *yA, const double *zA,
                             const double *xB, const double *yB, const double *zB,
                             double max_error, double pq[6], int32_t *iterations);
double dor_gjk(const double *a, int32_t na, const double *b, int32_t nb, double p[3], double q[3]);

/* ---- pair list (one triangle pair per element) -------------------------------- */
/* flags: PENALTY -> failed (0/1); PENALTY_ITER -> iterations; HYBRID_PAIR -> 1 if bf
 * was used; BF/GJK -> 0.  max_error is the penalty tolerance (reference: (epsA+epsB)/16). */
void dor_pairs(int32_t method, int64_t n, const double *a, const double *b, int64_t ld,
               double max_error, double *p, double *q, double *dist, uint8_t *flags,
               int32_t nthreads);

/* ---- particle-pair drivers ------------------------------------------------------ */
/* Returns the number of contacts; writes at most cap of them. */
int64_t dor_detect(int32_t driver,
                   const double *xA, const double *yA, const double *zA, int32_t nA,
                   double epsA, int32_t fricA, int32_t idA,
                   const double *xB, const double *yB, const double *zB, int32_t nB,
                   double epsB, int32_t fricB, int32_t idB,
                   dor_contact *out, int64_t cap, dor_stats *stats);

void dor_make_contact(double xPA, double yPA, double zPA, double epsA, int32_t idA,
                      double xPB, double yPB, double zPB, double epsB, int32_t idB,
                      int32_t friction, dor_contact *c);

/* ---- forces and dynamics ---------------------------------------------------------- */
typedef struct { double spring, damper, friction; } dor_material;

void dor_contacts_forces(const dor_contact *c, int64_t nc, double normal_sign,
                         const double posA[3], const double angA[3], const double linA[3], double massA,
                         const double posB[3], const double angB[3], const double linB[3], double massB,
                         const dor_material *mat, double force[3], double torque[3]);
void dor_expmap(double o1, double o2, double o3, double L[9]);
void dor_update_rotation(double ang[3], const double ref_ang[3], double rot[9], double step);
void dor_update_angular(double ref_ang[3], const double rot[9], const double inertia[9],
                        const double inverse[9], const double torque[3], double step);
void dor_update_vertex(double *x, double *y, double *z, double rx, double ry, double rz,
                       const double rot[9], const double pos[3], const double ref_pos[3]);

/* ---- whole time step ---------------------------------------------------------------- */
typedef struct {
  int32_t n_bodies;
  const int64_t *tri_offset;   /* [n_bodies+1] triangle offsets */
  double *x, *y, *z;           /* spatial SoA-tri vertices, 3 per triangle */
  const double *rx, *ry, *rz;  /* referential SoA-tri vertices */
  double *pos;                 /* [3n] spatial centre of mass */
  const double *ref_pos;       /* [3n] referential centre of mass */
  double *vel;                 /* [3n] linear velocity */
  double *ang;                 /* [3n] spatial angular velocity */
  double *ref_ang;             /* [3n] referential angular velocity */
  double *rot;                 /* [9n] orientation, column-major as in dynamics.cpp */
  const double *inertia;       /* [9n] */
  const double *inverse;       /* [9n] */
  const double *mass;          /* [n] (obstacles: +inf) */
  const double *eps;           /* [n] contact halo epsilon */
  const double *radius;        /* [n] bounding-sphere radius about pos */
  const uint8_t *friction;     /* [n] */
  const uint8_t *obstacle;     /* [n] */
} dor_scene;

typedef struct {
  double dt;
  double gravity[3];
  dor_material mat;
} dor_step_params;

typedef struct dor_sim dor_sim;
dor_sim *dor_sim_create(void);
void dor_sim_destroy(dor_sim *s);
/* Runs nsteps of the multiscale update order; returns the contact count of the last
 * detection (the contacts the next step's forces use). */
int64_t dor_sim_run(dor_sim *s, dor_scene *scene, const dor_step_params *prm, int32_t nsteps,
                    int64_t *contacts_per_step);
/* Copies out the contacts currently held (sorted by (master, slave, tri_a, tri_b)). */
int64_t dor_sim_contacts(const dor_sim *s, dor_contact *out, int64_t cap);

/* Sphere model (sphere.cpp, point.cpp).  dor_pt: closest point tq of triangle
 * (TP1,TP2,TP3) to c and its distance (point.cpp:11-210).  dor_sphere: sphere()
 * (sphere.cpp:29-77), diameters; 0 or 1 contact.  dor_sphere_mesh: sphereWithBarrierAB
 * (ba = 0: the sphere is A, the mesh B; sphere.cpp:79-140) or sphereWithBarrierBA (ba = 1;
 * sphere.cpp:142-201); triangle order.  dor_sphere_overlay: isSphereOverlayInContact
 * (sphere.cpp:203-218), radii. */
double dor_pt(const double TP1[3], const double TP2[3], const double TP3[3], const double c[3], double tq[3]);
int64_t dor_sphere(const double cA[3], double dA, double epsA, int32_t fricA, int32_t idA, const double cB[3],
                   double dB, double epsB, int32_t fricB, int32_t idB, dor_contact *out);
int64_t dor_sphere_mesh(int32_t ba, const double c[3], double d, double epsS, int32_t fricS, int32_t idS,
                        const double *x, const double *y, const double *z, int32_t nT, double epsM, int32_t fricM,
                        int32_t idM, dor_contact *out, int64_t cap);
int32_t dor_sphere_overlay(const double cA[3], double rA, const double cB[3], double rB);

/* Contact de-duplication (filter.cpp).  Contacts are given by their points x as 3 planes
 * of ld doubles and their (master, slave) ids; a segment is a maximal run of equal
 * (master, slave).  filterNewContacts (filter.cpp:80-101) within each segment, in order:
 * keep[i] = 1 unless an earlier kept contact of the segment lies within eps on every
 * coordinate (|dx| < eps).  filterOldContacts (filter.cpp:3-78, all three overloads):
 * keep[i] = 0 when any stored contact with the same (master, slave) lies within eps. */
void dor_filter_new(int64_t n, const double *x, int64_t ld, const int32_t *master, const int32_t *slave,
                    double eps, uint8_t *keep);
void dor_filter_old(int64_t ns, const double *xs, int64_t lds, const int32_t *ms, const int32_t *ss, int64_t nn,
                    const double *xn, int64_t ldn, const int32_t *mn, const int32_t *sn, double eps,
                    uint8_t *keep);

/* ---- the zoltan/ code path (zoltan_oracle.c) ------------------------------------------
 * Planar layouts: d, e, f, p, q hold 3 planes of ld doubles (plane k = coordinate k);
 * per-body vectors plane k of nb; triangles t: plane 3*v + k of ldt (v = 0..2 spatial,
 * 3..5 referential vertices). */
/* zoltan/bf.cpp:26-952 for one pair; returns 1 on its early return (pq untouched). */
int dzo_bf(const double *xA, const double *yA, const double *zA, const double *xB, const double *yB,
           const double *zB, double pq[6]);
/* bf(it, nt, ...) (declared at zoltan/bf.h:61-64): dzo_bf for i in [it, nt) */
void dzo_bf_soa(uint32_t it, uint32_t nt, const double a[3], const double b[3], const double c[3], const double *d,
                const double *e, const double *f, int64_t ld, double *p, double *q);
/* penalty(it, nt, ...), zoltan/penalty.cpp:27-209 */
void dzo_penalty(uint32_t it, uint32_t nt, const double a[3], const double b[3], const double c[3],
                 const double *d, const double *e, const double *f, int64_t ld, double *p, double *q);
/* hybrid(it, nt, ...), zoltan/hybrid.cpp:37-131 (it counts batches of 4) */
void dzo_hybrid(int32_t it, int32_t nt, const double a[3], const double b[3], const double c[3], const double *d,
                const double *e, const double *f, int64_t ld, double *p, double *q);
/* The same two with the penalty weight r moved by r_ulps units in the last place (test
 * hook: which results depend on the last bit of pow/log/log10); hybrid's mode 0 keeps the
 * reference's fallback decision, 1 never falls back, 2 always falls back. */
void dzo_penalty_shifted(uint32_t it, uint32_t nt, const double a[3], const double b[3], const double c[3],
                         const double *d, const double *e, const double *f, int64_t ld, double *p, double *q,
                         int32_t r_ulps);
void dzo_hybrid_shifted(int32_t it, int32_t nt, const double a[3], const double b[3], const double c[3],
                        const double *d, const double *e, const double *f, int64_t ld, double *p, double *q,
                        int32_t r_ulps, int32_t mode);
/* dynamics::update, euler, integrate (zoltan/dynamics.cpp:66-335) */
void dzo_update(int32_t nt, int32_t nb, double *t, int64_t ldt, const int32_t *pid, double *angular,
                double *linear, double *rotation, double *position, const double *inertia, const double *inverse,
                const double *mass, double *force, double *torque, double step);
void dzo_euler(int32_t nb, double *angular, const double *linear, double *rotation, double *position, double step);
void dzo_integrate(double step, const double lo[3], const double hi[3], int32_t nt, double *t, int64_t ldt,
                   double *v);
/* forces::force (zoltan/forces.cpp:48-205) on one process; contacts grouped by master:
 * [offset[i], offset[i+1]), fields as 3 planes (point, normal) or one (depth) of ldc. */
void dzo_force(int32_t nb, const int64_t *offset, const int32_t *slave, const double *point, const double *normal,
               const double *depth, int64_t ldc, const double *position, const double *angular, const double *linear,
               const double *mass, double *force, double *torque, const double gravity[3], double spring,
               double damper);

#ifdef __cplusplus
}
#endif
#endif
