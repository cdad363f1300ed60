/*
 * delta_b200.h -- C ABI of the B200 contact pipeline for triangulated particles.
 *
 * Plain pointers and sizes only.  Unless a function name ends in _host, every array
 * argument is a device pointer on the context's device; the caller owns all buffers.
 * Every call is asynchronous on the context's stream unless stated otherwise, and
 * returns a delta_status.  delta_last_error() gives a one-line description of the last
 * failure on the calling thread.
 *
 * Layouts
 *   pair list : a, b hold 9 planes of ld doubles; plane k = 3*vertex + coord, entry i
 *               is triangle pair i (the SoA pair-list shape of ispc_bf / ispc_pen,
 *               delta/contact/detection/bf.ispc:3, penalty.ispc:154).
 *               p, q hold 3 planes of ld doubles (closest points on A and on B).
 *   SoA-tri   : x, y, z hold 3 entries per triangle; triangle t of body i sits at
 *               3*(tri_offset[i]+t) .. +2 (ParticleRecord _xCoordinates; the argument
 *               shape of delta::contact::detection::bf, bf.h:65-81).
 */
#ifndef DELTA_B200_H
#define DELTA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  DELTA_OK = 0,
  DELTA_ERR_INVALID = 1,     /* bad argument (null pointer, negative size, unknown method) */
  DELTA_ERR_CUDA = 2,        /* a CUDA runtime call failed */
  DELTA_ERR_CAPACITY = 3,    /* an output buffer is too small; the needed size is returned */
  DELTA_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up */
  DELTA_ERR_NOMEM = 5,       /* device or pinned-host allocation failed */
  DELTA_ERR_UNSUPPORTED = 6  /* method/precision combination not built */
} delta_status;

/* Narrowphase methods. */
typedef enum {
  DELTA_BF = 0,            /* bfSolver, bf.cpp:217-1178: exact 9 edge-edge + 6 vertex-face */
  DELTA_PENALTY = 1,       /* penaltySolver(..., MaxError, bool& failed), penalty.cpp:278-432 */
  DELTA_PENALTY_ITER = 2,  /* penaltySolver(..., maxError, int& iterations), penalty.cpp:434-582 */
  DELTA_GJK = 3,           /* gjk(a,3,b,3,p,q), gjk.cpp:418-460 */
  DELTA_HYBRID_PAIR = 4,   /* penalty, bf when it reports failure (per pair) */
  DELTA_BF_CERT = 5        /* FP32 feature filter + FP64 evaluation of the certified
                              candidate features; equal to DELTA_BF in FP64 */
} delta_method;

typedef enum {
  DELTA_F64 = 0,  /* reference arithmetic in FP64, no FMA contraction */
  DELTA_F32 = 1   /* the same algorithm in FP32 (the reference's iREAL=float build) */
} delta_precision;

/* Particle-pair drivers (the functions Collision::collisionDetection switches over,
 * multiscale/dem/mappings/Collision.cpp:342-645). */
typedef enum {
  DELTA_DRV_BF = 0,                /* bf(),                          bf.cpp:47-148      */
  DELTA_DRV_PENALTY = 1,           /* penalty(),                     penalty.cpp:133-275 */
  DELTA_DRV_PENALTY_STAT = 2,      /* penaltyStat(),                 penalty.cpp:50-110  */
  DELTA_DRV_HYBRID_BATCH = 3,      /* hybridWithPerBatchFallBack(),  hybrid.cpp:357-487  */
  DELTA_DRV_HYBRID_TRIANGLE = 4,   /* hybridWithPerTriangleFallBack, hybrid.cpp:78-200   */
  DELTA_DRV_HYBRID_BATCH_STAT = 5, /* hybridBatchStat(),             hybrid.cpp:489-628  */
  DELTA_DRV_HYBRID_TRI_STAT = 6,   /* hybridTriangleStat(),          hybrid.cpp:202-336  */
  DELTA_DRV_GJK = 7,               /* gjk per triangle pair with bf()'s contact rule     */
  DELTA_DRV_BF_CERT = 8,           /* bf() contact set computed with DELTA_BF_CERT        */
  DELTA_DRV_BF_CULLED = 9,         /* bf() contact set: the certified driver's exact box
                                      culling, then FP64 bfSolver on the survivors        */
  DELTA_DRV_LEARNED = 10           /* the learned FP32 hybrid: the same culling, then per
                                      survivor 2 FP32 projection sweeps, the bfSolver
                                      feature they name in FP64, a separating-plane
                                      certificate at 1e-6 relative, and DELTA_BF_CERT for
                                      the pairs it does not certify; bf()'s contact rule on
                                      the FP64 distance, so the contact set is bf()'s
                                      except for pairs within 1e-6 of the threshold       */
} delta_driver;

typedef struct delta_ctx delta_ctx;

/* ---- context ---------------------------------------------------------------------- */
/* stream: a cudaStream_t (NULL = the legacy default stream).  The context owns its
 * scratch buffers and pinned staging memory. */
delta_status delta_create(delta_ctx **ctx, int device, void *stream);
delta_status delta_destroy(delta_ctx *ctx);
delta_status delta_set_stream(delta_ctx *ctx, void *stream);
/* Waits for the context's stream; DELTA_ERR_TIMEOUT when a tcgen05 GEMM's bounded wait
 * gave up since the last call. */
delta_status delta_synchronize(delta_ctx *ctx);
const char *delta_last_error(void);
const char *delta_version(void);
/* Number of kernel launches the library issued on this context so far. */
int64_t delta_launch_count(const delta_ctx *ctx);

/* ---- pair list -------------------------------------------------------------------- */
/* Closest points and distance for n independent triangle pairs.  max_error is the
 * penalty tolerance (the reference passes (epsA+epsB)/16).  flags (may be NULL):
 * PENALTY -> failed (0/1); PENALTY_ITER -> iterations on early exit, else 0;
 * HYBRID_PAIR -> 1 where bf ran; BF_CERT -> number of features evaluated in FP64;
 * BF/GJK -> 0.  Replaces the per-pair loops of bf()/penalty() (bf.cpp:95-118,
 * penalty.cpp:187-210) and ispc_bf / ispc_pen. */
delta_status delta_pairs_run(delta_ctx *ctx, int method, int precision, int64_t n, const double *a,
                             const double *b, int64_t ld, double max_error, double *p, double *q,
                             double *dist, uint8_t *flags);

/* Same with host buffers: copies the inputs to the device, runs, copies the results
 * back and synchronises.  Large host buffers are staged through pinned memory. */
delta_status delta_pairs_run_host(delta_ctx *ctx, int method, int precision, int64_t n, const double *a,
                                  const double *b, int64_t ld, double max_error, double *p, double *q,
                                  double *dist, uint8_t *flags);

/* Launch shape of the pair kernel of (method, precision) on this context: threads per
 * block (64, 128 or 256; the certified kernel and the FP64 bf kernel take 64 or 128) and
 * the grid cap in blocks per SM (0: no cap, one thread per pair).  No counterpart in the
 * reference (its SIMD width and OpenMP schedule are compile-time, bf.cpp:93-102). */
delta_status delta_set_pair_launch(delta_ctx *ctx, int method, int precision, int32_t threads,
                                   int32_t blocks_per_sm);

/* Autotuner: runs the pair kernel of (method, precision) over the given pairs (device
 * buffers, as delta_pairs_run) with each candidate launch shape, times them with CUDA
 * events, and keeps the fastest for this context.  Writes the choice and its time per
 * launch.  Synchronises.  (The reference's counterpart is the Peano grain-size oracle,
 * multiscale/sharedmemoryoracles.) */
delta_status delta_autotune_pairs(delta_ctx *ctx, int method, int precision, int64_t n, const double *a,
                                  const double *b, int64_t ld, double max_error, double *p, double *q,
                                  double *dist, uint8_t *flags, int32_t *threads_out, int32_t *blocks_per_sm_out,
                                  float *ms_out);

/* No counterpart in the reference.  delta_pairs_run_host for callers that must not let
 * the library allocate device memory: a host whose own pooling allocator owns the GPU
 * memory, or an allocation-free latency-bound loop.  Inputs and outputs are staged in one
 * fixed device array built into the library (DELTA_NOALLOC_MAX_PAIRS pairs, 201 bytes
 * each: 65,863,680 bytes = 62.8 MiB, held on every GPU that loads the library until the
 * process exits); no cudaMalloc, cudaFree or allocating library routine is called.  n
 * above the maximum returns DELTA_ERR_CAPACITY.  The launch shape is the context's, as
 * for delta_pairs_run_host.  The first call on a device looks the array's device address
 * up (and may make the driver load the library module there); the address is kept for
 * the device, so do not use this entry point across a cudaDeviceReset.  All calls on a
 * device share the array and leave their data in it; calls that overlap on the GPU race.
 * Synchronises the context's stream. */
#define DELTA_NOALLOC_MAX_PAIRS 327680
delta_status delta_pairs_run_host_noalloc(delta_ctx *ctx, int method, int precision, int64_t n, const double *a,
                                          const double *b, int64_t ld, double max_error, double *p, double *q,
                                          double *dist, uint8_t *flags);

/* ---- particle pairs ------------------------------------------------------------------ */
/* Triangulated bodies in SoA-tri layout (device arrays). */
typedef struct {
  int32_t n_bodies;
  const int64_t *tri_offset;  /* [n_bodies+1] first triangle of each body */
  const double *x, *y, *z;    /* [3*tri_offset[n_bodies]] vertices, 3 per triangle */
  const double *eps;          /* [n_bodies] contact halo epsilon */
  const uint8_t *friction;    /* [n_bodies] friction flag */
  const int32_t *id;          /* [n_bodies] global particle id written to master/slave */
} delta_meshes;

/* Contacts in SoA (device arrays of `capacity` entries; x, normal, P, Q hold 3 planes of
 * `capacity`).  One entry per struct contactpoint (contactpoint.h:42-103) plus the
 * triangle indices that produced it. */
typedef struct {
  int64_t capacity;
  double *x, *normal, *P, *Q;
  double *depth, *eps_total;
  int32_t *master, *slave, *tri_a, *tri_b, *penetration;
  uint8_t *friction;
} delta_contacts;

/* Statistics of the instrumented drivers (penalty.cpp:29-48, hybrid.cpp:27-56). */
typedef struct {
  int64_t newton_hist[17];
  int64_t penalty_fails;
  int64_t batch_fails;
  int64_t batch_size;
  double batch_error;
} delta_stats;

/* Runs `driver` on every candidate body pair (pair_a[k], pair_b[k]) (device arrays of
 * n_pairs) and writes the contacts, ordered by (pair k, A triangle, B triangle) -- the
 * serial order of the reference drivers.  Each body must have fewer than 65536
 * triangles.  *n_out (host) receives the contact count; when it exceeds
 * out->capacity, nothing past the capacity is written and DELTA_ERR_CAPACITY is
 * returned.  stats (host, may be NULL) is overwritten with this call's statistics.
 * Synchronises the context's stream.  Drop-in for bf() / penalty() / penaltyStat() /
 * hybridWith{PerBatch,PerTriangle}FallBack() / hybrid{Batch,Triangle}Stat() called per
 * candidate pair by Collision::collisionDetection (Collision.cpp:342-645), with the
 * contact lists of all pairs concatenated. */
delta_status delta_detect(delta_ctx *ctx, int driver, int precision, const delta_meshes *meshes,
                          const int32_t *pair_a, const int32_t *pair_b, int64_t n_pairs,
                          const delta_contacts *out, int64_t *n_out, delta_stats *stats);

/* ---- forces, integration, broadphase, time step -------------------------------------- */
/* Rigid bodies (device arrays).  Per-body vectors are SoA planes: component k of body i
 * is at [k*n_bodies + i]; rot is the 3x3 orientation stored column-major as in
 * delta/dynamics/dynamics.cpp (rot[(3*col+row)*n_bodies + i]). */
typedef struct {
  int32_t n_bodies;
  const int64_t *tri_offset;   /* [n_bodies+1] */
  const int32_t *tri_body;     /* [n_triangles] owner body of each triangle */
  double *x, *y, *z;           /* spatial vertices, SoA-tri */
  const double *rx, *ry, *rz;  /* referential vertices, SoA-tri */
  double *pos;                 /* [3n] spatial centre of mass */
  const double *ref_pos;       /* [3n] referential centre of mass */
  double *vel;                 /* [3n] linear velocity */
  double *ang;                 /* [3n] spatial angular velocity */
  double *ref_ang;             /* [3n] referential angular velocity */
  double *rot;                 /* [9n] orientation */
  const double *inertia;       /* [9n] */
  const double *inverse;       /* [9n] */
  const double *mass;          /* [n] (obstacles: +inf) */
  const double *eps;           /* [n] contact halo epsilon */
  const double *radius;        /* [n] bounding-sphere radius about pos */
  const uint8_t *friction;     /* [n] */
  const uint8_t *obstacle;     /* [n] obstacles never move */
} delta_scene;

typedef struct {
  double dt;
  double gravity[3];  /* added to the velocity as dt*gravity (MoveParticles.cpp:73 uses 9.8 along -y) */
  double spring;      /* SPRING, forces.cpp:11-14 */
  double damper;      /* DAMPER */
  double friction;    /* FRICTION */
} delta_step_params;

/* Per-body force and torque from contacts sorted by (master, slave, tri_a, tri_b) with
 * master/slave = body indices: for each body, the contributions of its partners in
 * ascending partner order, each partner's contacts summed in list order
 * (Collision::touchVertexFirstTime, Collision.cpp:1060-1101 -> getContactsForces,
 * forces.cpp:291-396; the slave side uses the inverted normal, Collision.cpp:176-184).
 * force, torque: [3n] planes; has_contact: [n] (1 where the body has a partner). */
delta_status delta_forces(delta_ctx *ctx, const delta_scene *scene, const delta_contacts *contacts,
                          int64_t n_contacts, const delta_step_params *params, double *force,
                          double *torque, uint8_t *has_contact);

/* v += dt*F/m and updateAngular (dynamics.cpp:140-213) for bodies with a contact
 * (Collision.cpp:1105-1115), then for every non-obstacle body v += dt*g, x += dt*v,
 * updateRotationMatrix (dynamics.cpp:104-138) and updateVertices (dynamics.cpp:215-242)
 * (MoveParticles.cpp:63-112). */
delta_status delta_integrate(delta_ctx *ctx, const delta_scene *scene, const delta_step_params *params,
                             const double *force, const double *torque, const uint8_t *has_contact);

/* getContactsForces (forces.cpp:291-396) for n_groups calls at once.  Group g is one call:
 * the contacts [offset[g], offset[g+1]) of `contacts` (x, normal, depth and friction are
 * read; the normal as stored for body A), body A's and body B's centre, spatial angular
 * velocity and linear velocity (pos_a, ang_a, lin_a, ... : 3 planes of n_groups) and
 * masses (mass_a, mass_b: n_groups).  force and torque (3 planes of n_groups) accumulate
 * onto their inputs contact by contact, as the reference adds into its force[3] and
 * torque[3].  params: spring, damper, friction (SPRING, DAMPER, FRICTION, forces.cpp:11-21;
 * a sphere contact, isSphere, is springSphere's formula with SSPRING, SDAMPER and
 * SFRICTIONGOLD, forces.cpp:227-289); dt and gravity are not used. */
delta_status delta_contact_forces(delta_ctx *ctx, int64_t n_groups, const int64_t *offset,
                                  const delta_contacts *contacts, const double *pos_a, const double *ang_a,
                                  const double *lin_a, const double *mass_a, const double *pos_b,
                                  const double *ang_b, const double *lin_b, const double *mass_b,
                                  const delta_step_params *params, double *force, double *torque);
/* updateAngular (dynamics.cpp:140-213) of n bodies: ref_ang [3n] in/out, rot [9n],
 * inertia [9n], inverse [9n], torque [3n]. */
delta_status delta_update_angular(delta_ctx *ctx, int32_t n, double *ref_ang, const double *rot,
                                  const double *inertia, const double *inverse, const double *torque, double step);
/* updateRotationMatrix (dynamics.cpp:104-138) of n bodies: rot [9n] in/out, the spatial
 * angular velocity ang [3n] out, from ref_ang [3n]. */
delta_status delta_update_rotation(delta_ctx *ctx, int32_t n, double *ang, const double *ref_ang, double *rot,
                                   double step);
/* updateVertices (dynamics.cpp:215-242) of n_vertices vertices: vertex v gets
 * pos + R (r - ref_pos) of its body body[v] (body may be NULL when n_bodies == 1);
 * rot [9 n_bodies], pos, ref_pos [3 n_bodies]. */
delta_status delta_update_vertices(delta_ctx *ctx, int64_t n_vertices, const int32_t *body, int32_t n_bodies,
                                   double *x, double *y, double *z, const double *rx, const double *ry,
                                   const double *rz, const double *rot, const double *pos, const double *ref_pos);

/* Candidate body pairs (a < b, not both obstacles) whose bounding spheres, grown by the
 * two epsilons, overlap; sorted by (a, b).  A superset of the pairs that can hold a
 * contact (replaces the Peano grid traversal + isSphereOverlayInContact precheck,
 * Collision.cpp:893-958, sphere.cpp:203-218).  *n_out receives the count; beyond
 * `capacity` DELTA_ERR_CAPACITY.  Synchronises. */
delta_status delta_broadphase(delta_ctx *ctx, const delta_scene *scene, int32_t *pair_a, int32_t *pair_b,
                              int64_t capacity, int64_t *n_out);

/* A simulation: the scene plus the contacts of the last detection.  One step follows
 * the multiscale order: forces from the previous detection's contacts, velocity and
 * angular update, move, then broadphase and narrowphase with `driver`.  Within a call,
 * a step updates the vertices (updateVertices) of only the bodies of its candidate pairs,
 * the only vertices the narrowphase reads (the certified driver updates none: it forms
 * the vertices it reads from the bodies' poses with the same arithmetic); all vertices
 * are updated at the end of the call, so the scene's vertex arrays equal those of a
 * per-step full update whenever a call returns.  The scene's buffers stay the caller's;
 * the simulation reads the obstacles' vertices (their boxes) and the reference vertices
 * and centres (each body's reach) once, at creation, so those must not change while it
 * exists (in the reference they never do). */
typedef struct delta_sim delta_sim;
delta_status delta_sim_create(delta_ctx *ctx, const delta_scene *scene, int driver, delta_sim **out);
delta_status delta_sim_step(delta_sim *sim, const delta_step_params *params, int32_t nsteps,
                            int64_t *contacts_per_step /* host [nsteps] or NULL */);
/* Same steps as delta_sim_step, recorded once as a CUDA graph (every kernel of a step,
 * fixed-capacity buffers, counts kept on the device) and replayed nsteps times without
 * host synchronisation.  The first call sizes the buffers from an observed detection.
 * The replayed step takes its candidate pairs from a skin list: the sorted pairs within
 * reach + skin (skin = 1/32 of a broadphase cell), filtered each step with the exact
 * candidate test; a conditional node of the graph rebuilds the list at the start of each
 * call and in any step where a moving body has moved more than skin/2 since the last
 * build, so the candidates, and their order, are those of delta_sim_step's search.
 * A capacity overflow in a replayed step freezes the state after that step's
 * integration; the host then repeats that detection with larger buffers, records the
 * graph again and continues, so results equal delta_sim_step's bit for bit.  The buffers
 * and the recorded graph are kept from call to call while the current contacts fit; the
 * graph is recorded again whenever params change. */
delta_status delta_sim_step_graph(delta_sim *sim, const delta_step_params *params, int32_t nsteps,
                                  int64_t *contacts_per_step /* host [nsteps] or NULL */);
/* Capacities (candidate pairs, contacts) of the graph buffers for the next
 * delta_sim_step_graph call instead of the observed-size default; overflows still
 * recover as described above. */
delta_status delta_sim_set_graph_capacity(delta_sim *sim, int64_t pair_capacity, int64_t contact_capacity);
/* The graph step's skin list: the skin distance (0: no list, the step searches the grid),
 * the list's capacity (0 before the first graph call) and the builds run inside graph
 * replays so far. */
delta_status delta_sim_skin_stats(delta_sim *sim, double *skin, int64_t *capacity, int64_t *rebuilds);
/* Launch shapes of the culled drivers' two kernels (DELTA_DRV_BF_CERT, DELTA_DRV_BF_CULLED,
 * DELTA_DRV_LEARNED): the culling kernel's and the survivors' solver's resident blocks per
 * SM (0 = as many as fit; larger values are clamped to what fits).  They belong to the
 * context and apply to every detection it runs; a simulation's recorded graph is recorded
 * again with them on its next delta_sim_step_graph call. */
delta_status delta_set_cull_launch(delta_ctx *ctx, int32_t cull_blocks_per_sm, int32_t survivor_blocks_per_sm);
/* Times the detection of the simulation's current state (the same candidate pairs, reps
 * runs after one warm-up, median) under every launch shape of the culled driver's two
 * kernels that fits, keeps the fastest in the context (delta_set_cull_launch) and writes
 * it to choice[0..1], its median time in ms to *ms_out (may be NULL).  The state is not
 * changed (the current contacts are detected again, alike); the counters are kept.  For
 * the other drivers nothing is tuned: choice = {0, 0}. */
delta_status delta_sim_autotune(delta_sim *sim, int32_t reps, int32_t choice[2], float *ms_out);
/* Copies the current contacts into out (device); *n_out gets their number. */
delta_status delta_sim_contacts(delta_sim *sim, const delta_contacts *out, int64_t *n_out);
/* Totals since creation: [0] steps, [1] candidate body pairs, [2] triangle pairs of the
 * candidates (sum of nA*nB: the pairs the reference tests, Collision.cpp:652), [3]
 * triangle pairs the narrowphase solver ran on (after exact box culling for BF_CERT). */
delta_status delta_sim_counters(const delta_sim *sim, int64_t out[4]);
delta_status delta_sim_destroy(delta_sim *sim);

/* ---- sphere model ----------------------------------------------------------------------
 * sphere.cpp / point.cpp: particles as spheres (the reference's cheap baseline and halo
 * precheck).  Contacts use the same record as the mesh path (contactpoint.cpp:116-155),
 * tri_a = -1, tri_b = the mesh triangle (or -1); they equal the reference's bit for bit.
 * The forces of sphere contacts are delta_forces' with the sphere constants (springSphere,
 * forces.cpp:227-253, is spring's formula with SSPRING and SDAMPER; the sphere friction
 * uses SFRICTIONGOLD). */
typedef struct {
  int64_t n;
  const double *centre;     /* [3][n] planes x, y, z */
  const double *diameter;   /* [n] (the reference passes diameters) */
  const double *eps;        /* [n] */
  const uint8_t *friction;  /* [n] */
  const int32_t *id;        /* [n] global particle id written to master/slave */
} delta_spheres;
/* sphere() (sphere.cpp:29-77) for the sphere pairs (pair_a[k], pair_b[k]): at most one
 * contact per pair, written in pair order.  *n_out = the number of contacts; beyond
 * out->capacity DELTA_ERR_CAPACITY.  Synchronises. */
delta_status delta_sphere_contacts(delta_ctx *ctx, const delta_spheres *spheres, const int32_t *pair_a,
                                   const int32_t *pair_b, int64_t n_pairs, const delta_contacts *out,
                                   int64_t *n_out);
/* sphereWithBarrierAB (sphere_is_b = 0: sphere.cpp:79-140) or sphereWithBarrierBA
 * (sphere_is_b = 1: sphere.cpp:142-201) for (sphere[k], mesh body[k]): one contact per
 * triangle of the body within the halo, in (pair, triangle) order.  Synchronises. */
delta_status delta_sphere_mesh_contacts(delta_ctx *ctx, const delta_spheres *spheres, const delta_meshes *meshes,
                                        const int32_t *sphere, const int32_t *body, int64_t n_pairs,
                                        int sphere_is_b, const delta_contacts *out, int64_t *n_out);
/* isSphereOverlayInContact (sphere.cpp:203-218) for each pair: centre [3][ld], radius [n]
 * (the values the caller passes as radii); overlap [n_pairs] = 1 when |cA - cB| <= rA + rB. */
delta_status delta_sphere_overlap(delta_ctx *ctx, const double *centre, int64_t ld, const double *radius,
                                  const int32_t *pair_a, const int32_t *pair_b, int64_t n_pairs, uint8_t *overlap);

/* ---- the zoltan/ code path -------------------------------------------------------------
 * The reference's second front end (zoltan/) keeps the system as structure-of-arrays and
 * calls the narrowphase with one triangle against a list.  These entry points keep those
 * argument lists: the reference's pointer arrays become arrays of device pointers
 * (d[k] = coordinate k of every list entry; t[v][k] = coordinate k of vertex v of every
 * triangle, v = 0..2 spatial and 3..5 referential); a, b, c, lo, hi and gravity are host
 * arrays of 3 doubles.  FP64 in the reference's operation order; the penalty weights use
 * pow/log/log10 (CUDA's, which can differ from the host C library's in the last bit).
 * Asynchronous on the context's stream. */

/* bf(it, nt, A, B, C, D, E, F, P, Q), declared at zoltan/bf.h:61-64 (the reference defines
 * only the per-pair form, zoltan/bf.cpp:26-952): for i in [it, nt), the closest points of
 * triangle ABC and triangle (D[i], E[i], F[i]) with zoltan/bf.cpp's arithmetic and its
 * differences from delta's bfSolver (early return on a zero cross product, leaving P[i],
 * Q[i] untouched; no break after case 1 of either switch). */
delta_status delta_zoltan_bf(delta_ctx *ctx, uint32_t it, uint32_t nt, const double a[3], const double b[3],
                             const double c[3], const double *const d[3], const double *const e[3],
                             const double *const f[3], double *const p[3], double *const q[3]);
/* penalty(it, nt, ...), zoltan/penalty.cpp:27-209: 5 quasi-Newton steps per entry, delta
 * = 0.1 tr(H) (multiplied by r before every step for entries i >= 4, as the reference's
 * test `i < 4` reads the list index), r = lambda 10^(ln lambda + 14). */
delta_status delta_zoltan_penalty(delta_ctx *ctx, uint32_t it, uint32_t nt, const double a[3], const double b[3],
                                  const double c[3], const double *const d[3], const double *const e[3],
                                  const double *const f[3], double *const p[3], double *const q[3]);
/* hybrid(it, nt, ...), zoltan/hybrid.cpp:37-131: batches k in [it, nt/4) of entries
 * 4k..4k+3 (it counts batches; entries past the last full batch are not visited); 7
 * penalty steps per entry; when the batch's mean error exceeds 1e-8, every entry of the
 * batch gets the points of the segment-triangle / vertex-face / edge-edge bf of
 * hybrid.cpp:646-886 applied to the batch's last entry (the reference's serial loop reuses
 * the last D, E, F), with that bf's own quirks (SMALL_NUM 1e-8; Q's y and z of an
 * edge-edge point start from p4's x, hybrid.cpp:436-437). */
delta_status delta_zoltan_hybrid(delta_ctx *ctx, int32_t it, int32_t nt, const double a[3], const double b[3],
                                 const double c[3], const double *const d[3], const double *const e[3],
                                 const double *const f[3], double *const p[3], double *const q[3]);
/* dynamics::update, zoltan/dynamics.cpp:66-250 (loba and rank unused on one GPU): per body,
 * the half-step angular update with expmap, v += (step/m) force, rotation *= expmap(step
 * O), x += step v, and force and torque zeroed; then every triangle's spatial vertices
 * t[0..2] from its referential ones t[3..5] and its body pid[i].  angular[0..2] is the
 * referential angular velocity, angular[3..5] the spatial one; position[0..2] the centre,
 * position[3..5] the referential centre. */
delta_status delta_zoltan_update(delta_ctx *ctx, int32_t nt, int32_t nb, double *const t[6][3], const int32_t *pid,
                                 double *const angular[6], double *const linear[3], double *const rotation[9],
                                 double *const position[6], const double *const inertia[9],
                                 const double *const inverse[9], const double *mass, double *const force[3],
                                 double *const torque[3], double step);
/* dynamics::euler, zoltan/dynamics.cpp:252-297 */
delta_status delta_zoltan_euler(delta_ctx *ctx, int32_t nb, double *const angular[6], const double *const linear[3],
                                double *const rotation[9], double *const position[6], double step);
/* dynamics::integrate, zoltan/dynamics.cpp:299-335: t[0..2] += step v per triangle; a
 * velocity component flips for every vertex coordinate outside [lo, hi]. */
delta_status delta_zoltan_integrate(delta_ctx *ctx, double step, const double lo[3], const double hi[3], int32_t nt,
                                    double *const t[3][3], double *const v[3]);
/* forces::force, zoltan/forces.cpp:48-205, on one GPU (every body is this rank's, nothing
 * to migrate): the reference's std::vector<contactpoint> conpnt[nb] becomes contacts
 * grouped by master body, body i's at [offset[i], offset[i+1]) of n_contacts, with the
 * slave id (contactpoint pid[1]), point, normal and depth.  force and torque accumulate
 * onto their inputs in the serial loop's order: per master i, each contact adds granular's
 * f = (spring depth + damper sqrt(spring m_red) (v_ij . n)) n to i and -f to the slave,
 * with their torques about each body's centre, then i gets mass_i gravity.  spring and
 * damper are material::iparam[SPRING/DAMPER][GRANULAR] (zoltan/delta.cpp:69-70 sets 1e2,
 * 1).  Contacts whose slave is not in [0, nb) add nothing.  Uses context scratch. */
delta_status delta_zoltan_force(delta_ctx *ctx, int32_t nb, const int64_t *offset, const int32_t *slave,
                                int64_t n_contacts, const double *const point[3], const double *const normal[3],
                                const double *depth, const double *const position[6],
                                const double *const angular[6], const double *const linear[3], const double *mass,
                                double *const force[3], double *const torque[3], const double gravity[3],
                                double spring, double damper);

/* ---- on-disk formats ------------------------------------------------------------------
 * The legacy ASCII VTK snapshot of all triangles, as writeGeometryToVTK writes it
 * (delta/core/io/write.cpp:226-306: file path + "geometry_<step>.vtk", POINTS at %.5f,
 * one triangle cell per three points, CELL_TYPES 5).  _host takes host arrays; the device
 * form copies the meshes back first (synchronises). */
delta_status delta_write_vtk_host(const char *path, int32_t step, int32_t n_bodies, const int64_t *tri_offset,
                                  const double *x, const double *y, const double *z);
delta_status delta_write_vtk(delta_ctx *ctx, const char *path, int32_t step, const delta_meshes *meshes);
/* writeGeometryToVTKVTK (delta/core/io/write.cpp:10-70) without the VTK library:
 * path + "geometry_<step>.vtu", an ASCII VTK XML unstructured grid of the n particle
 * centres (centre: 3 planes of n; Float32 points, as vtkPoints stores them), point data
 * "direction" = the linear velocity (3 planes of n) and "epsilon" (the reference's second
 * SetScalars call replaces its "radius"), no cells.  Host arrays. */
delta_status delta_write_vtu_host(const char *path, int32_t step, int64_t n, const double *centre,
                                  const double *velocity, const double *eps);
/* The same for a simulation's bodies (centre, velocity, epsilon). */
delta_status delta_sim_write_vtu(delta_sim *sim, const char *path, int32_t step);
/* The snapshot of a simulation's current vertices (obstacles included). */
delta_status delta_sim_write_vtk(delta_sim *sim, const char *path, int32_t step);
/* The .mbfcp scene reader (readmbfcp, delta/core/io/read.cpp:345-546): the material block's
 * friction, spring, dashpot, density and gravity (parsed with std::stof at the reference's
 * fixed offsets), the BODIES count, and every SPHERES body as (id, centre, radius) with the
 * reference's fixed-offset fields.  Host memory; *n_out = the number of spheres, beyond
 * capacity DELTA_ERR_CAPACITY; a malformed field gives DELTA_ERR_INVALID. */
typedef struct {
  int32_t *id;      /* [capacity] */
  double *centre;   /* [capacity][3] */
  double *radius;   /* [capacity] */
  int32_t bodies;   /* the BODIES: count */
  int32_t has_materials;
  double friction, spring, dashpot, density, gravity[3];
} delta_mbfcp;
delta_status delta_read_mbfcp(const char *filename, delta_mbfcp *out, int64_t capacity, int64_t *n_out);

/* ---- contact de-duplication ----------------------------------------------------------
 * filter.cpp (the reference defines these; its time step does not call them).  A run is a
 * maximal sequence of contacts with equal (master, slave), i.e. one particle pair's
 * contacts as delta_detect returns them.  keep [n] receives 1 for the contacts that stay.
 * eps is the reference's 0.0001 unless given otherwise; two contacts are near when
 * |x_a - x_b| < eps on every coordinate (FP64). */
/* filterNewContacts (filter.cpp:80-101) on every run: a contact stays unless an earlier
 * contact of its run that stayed is near it. */
delta_status delta_filter_new_contacts(delta_ctx *ctx, const delta_contacts *contacts, int64_t n, double eps,
                                       uint8_t *keep);
/* filterOldContacts (filter.cpp:3-78, all three overloads): a new contact stays unless a
 * stored contact of the same (master, slave) is near it.  Any order of either list. */
delta_status delta_filter_old_contacts(delta_ctx *ctx, const delta_contacts *stored, int64_t n_stored,
                                       const delta_contacts *fresh, int64_t n_fresh, double eps, uint8_t *keep);

/* ---- learned warm start ----------------------------------------------------------------
 * No counterpart in the reference.  A small MLP (18 -> 128 -> 128 -> 128 -> 4, GELU, BF16
 * weights and activations, FP32 accumulation) maps a canonicalised triangle pair to the
 * four barycentric weights that penaltySolver iterates on (x0, x1: P = A0 + x0 (A1-A0) +
 * x1 (A2-A0); x2, x3: Q on B likewise), which the reference starts at 0.33
 * (penalty.cpp:353-356).  These entry points are the network's training and inference
 * steps; row-major matrices, BF16 arrays passed as void* (2 bytes per element). */

/* Offsets (in elements) of W1 [128][32], b1, W2 [128][128], b2, W3, b3, W4 [4][128], b4 in
 * the flat parameter array, and [8] its length.  The FP32 master copy and the BF16 copy
 * share this layout; W1's columns 18..31 multiply zero features. */
delta_status delta_mlp_layout(int64_t offsets[9]);
/* Inference: the features kernel, then the four layers in one kernel on the mma.sync
 * path, into x0 [n][4] (FP32).  params is the FP32 array (biases are read from it),
 * params_bf16 the BF16 copy (weights); both x0 and params_bf16 16-byte aligned.  Equal bit
 * for bit to delta_mlp_features + delta_gemm_bf16 + delta_mlp_bias_act layer by layer. */
delta_status delta_mlp_infer(delta_ctx *ctx, int64_t n, const double *a, const double *b, int64_t ld,
                             const float *params, const void *params_bf16, float *x0);
/* Network engines of the learned hybrid (delta_pairs_run_learned) and of the training
 * GEMM (delta_gemm_bf16): the 5th-generation tensor cores (tcgen05 MMAs, TMEM
 * accumulators; the default) or the warp-level mma.sync path. */
#define DELTA_MLP_TCGEN05 0
#define DELTA_MLP_MMA_SYNC 1
delta_status delta_mlp_set_engine(delta_ctx *ctx, int engine);
/* delta_mlp_infer on the 5th-generation tensor cores (tcgen05 MMAs with TMEM
 * accumulators): same network and features, FP32 accumulation in a different order, so
 * x0 agrees with delta_mlp_infer to BF16 rounding rather than bit for bit.  params_bf16 and
 * x0 16-byte aligned.  Synchronises; DELTA_ERR_TIMEOUT if a bounded wait for the tensor
 * cores gave up (x0 is then incomplete). */
delta_status delta_mlp_infer_tcgen05(delta_ctx *ctx, int64_t n, const double *a, const double *b, int64_t ld,
                                     const float *params, const void *params_bf16, float *x0);
/* Test of the failure path of delta_mlp_infer_tcgen05 (no counterpart in the reference):
 * the kernel withholds the first layer's MMAs and commit, so its bounded wait for the
 * tensor cores runs out after `polls` polls (1 .. 2^22) with nothing in flight; the kernel
 * frees its TMEM and returns.  Expected result: DELTA_ERR_TIMEOUT, the context still
 * usable; x0 is left unspecified.  Same arguments as delta_mlp_infer_tcgen05, n > 0. */
delta_status delta_mlp_infer_tcgen05_wait_test(delta_ctx *ctx, int64_t n, const double *a, const double *b,
                                               int64_t ld, const float *params, const void *params_bf16, float *x0,
                                               uint32_t polls);
/* Canonical features: triangle A's frame (origin at its centroid, x along A1-A0, z along
 * its normal, unit = its longest edge), the six vertices in that frame as 18 BF16 values
 * padded with zeros to rows of 32 (features_bf16 [n][32]).  With p, q (closest points,
 * pair-list planes) also the targets [n][4] (barycentric weights of p on A and q on B).
 * features_bf16 and targets 16-byte aligned.
 * valid [n] (optional) is 0 for pairs with a degenerate triangle. */
delta_status delta_mlp_features(delta_ctx *ctx, int64_t n, const double *a, const double *b, int64_t ld,
                                const double *p, const double *q, void *features_bf16, float *targets,
                                uint8_t *valid);
/* C[M][N] (+)= op(A) op(B): A is [M][K] (trans_a 0) or [K][M]; B is [K][N] (trans_b 0)
 * or [N][K]; BF16 operands on the tensor cores, FP32 C.  On the context's engine: tcgen05
 * (the default: 128 x 128 output tiles, M=128 MMAs from shared memory into a TMEM
 * accumulator that sums the CTA's whole K range; with split_k > 1 the K splits write
 * partial tiles that one more kernel adds in split order, without atomics; a bounded wait
 * that gives up sets the output to NaN and makes the next delta_synchronize return
 * DELTA_ERR_TIMEOUT) or mma.sync (split_k > 1 accumulates with atomics). */
delta_status delta_gemm_bf16(delta_ctx *ctx, int M, int N, int K, const void *A, int lda, int trans_a,
                             const void *B, int ldb, int trans_b, float *C, int ldc, int accumulate, int split_k);
/* Z[M][N] += bias; H_bf16 (optional) = bf16(GELU(Z)) (tanh form) or bf16(Z) when gelu_on is 0. */
delta_status delta_mlp_bias_act(delta_ctx *ctx, int64_t M, int N, float *Z, const float *bias, void *H_bf16,
                                int gelu_on);
/* Mean-squared error over rows with valid != 0: dY_bf16 [M][4] = 2 (Y-T) inv_n, and
 * *loss += sum (Y-T)^2 inv_n (inv_n = 1 / number of valid rows). */
delta_status delta_mlp_mse(delta_ctx *ctx, int64_t M, const float *Y, const float *T, const uint8_t *valid,
                           float inv_n, void *dY_bf16, float *loss);
/* dZ_bf16 = bf16(dH * GELU'(Z)). */
delta_status delta_mlp_act_grad(delta_ctx *ctx, int64_t M, int N, const float *dH, const float *Z, void *dZ_bf16);
/* db[N] += column sums of dZ_bf16 [M][N]. */
delta_status delta_mlp_colsum(delta_ctx *ctx, int64_t M, int N, const void *dZ_bf16, float *db);
/* One Adam step (bias-corrected, step >= 1) on FP32 master weights w with moments m, v;
 * w_bf16 (optional) receives the BF16 copy. */
delta_status delta_adam(delta_ctx *ctx, int64_t n, float *w, const float *g, float *m, float *v, float lr, float b1,
                        float b2, float eps, int64_t step, void *w_bf16);
delta_status delta_to_bf16(delta_ctx *ctx, int64_t n, const float *x, void *y_bf16);
/* penaltySolver(..., maxError, int& iterations) (penalty.cpp:434-582, FP64 reference
 * arithmetic) started from x0 [n][4] instead of 0.33 (x0 NULL: 0.33).  iterations [n]
 * gets the iteration count, 16 when the step-size test never passed. */
delta_status delta_penalty_warm(delta_ctx *ctx, int64_t n, const double *a, const double *b, int64_t ld,
                                const float *x0, double max_error, double *p, double *q, double *dist,
                                uint8_t *iterations);
/* The learned solver.  From x0 [n][4] (16-byte aligned; NULL: the centroids), `sweeps`
 * FP32 alternating closest-point projections between the triangles; then `features`
 * bfSolver features are evaluated in FP32: 3 = those the projections name (B's nearest
 * vertex against face A, A's nearest vertex against face B, the nearest edge pair), 7 = all
 * six vertex-face features and that edge pair, 11 = all six vertex-face features and the
 * six edge pairs containing A's or B's nearest edge, 15 = all.  The one bfSolver's rule
 * (bf.cpp:1102) picks among them is evaluated in FP64 with the reference arithmetic: p, q,
 * dist.
 * Then an FP64 separating-plane certificate: with r = p - q, every plane normal to r
 * bounds the distance below by min_i r.A_i/|r| - max_j r.B_j/|r|; certified [n] is 1 when
 * |r| exceeds that bound by at most rel_tol |r|, so dist is within rel_tol of the true
 * distance.  Intersecting triangles are never certified; uncertified pairs are for
 * DELTA_BF_CERT. */
delta_status delta_learned_refine(delta_ctx *ctx, int64_t n, const double *a, const double *b, int64_t ld,
                                  const float *x0, int32_t sweeps, int32_t features, double rel_tol, double *p,
                                  double *q, double *dist, uint8_t *certified);
/* The learned hybrid narrowphase over a pair list (n < 2^32): delta_mlp_infer (skipped
 * when params and params_bf16 are NULL: the same solver from the centroids), then
 * delta_learned_refine, which lists the uncertified pairs on the device, then
 * DELTA_BF_CERT over that list.  Every distance is within rel_tol of FP64 bfSolver's and
 * every listed pair equals bfSolver bit for bit.  flags [n] (optional): 1 certified,
 * 2 solved exactly.  n_fallback (host, optional) receives the number of listed pairs and
 * makes the call synchronise (and report a tensor-core time-out of the network as
 * DELTA_ERR_TIMEOUT); otherwise asynchronous.  The network runs on the context's engine
 * (delta_mlp_set_engine). */
delta_status delta_pairs_run_learned(delta_ctx *ctx, int64_t n, const double *a, const double *b, int64_t ld,
                                     const float *params, const void *params_bf16, int32_t sweeps, int32_t features,
                                     double rel_tol, double *p, double *q, double *dist, uint8_t *flags,
                                     int64_t *n_fallback);
/* Same with host pair buffers (a, b, p, q, dist, flags; row pitch ld): copies in, runs,
 * copies out and synchronises.  params / params_bf16 stay device pointers (the network
 * is loaded once). */
delta_status delta_pairs_run_learned_host(delta_ctx *ctx, int64_t n, const double *a, const double *b, int64_t ld,
                                          const float *params, const void *params_bf16, int32_t sweeps,
                                          int32_t features, double rel_tol, double *p, double *q, double *dist,
                                          uint8_t *flags, int64_t *n_fallback);

#ifdef __cplusplus
}
#endif
#endif
