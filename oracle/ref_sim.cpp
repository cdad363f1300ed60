// ref_sim.cpp -- a whole time step driven by the reference's own functions (bf(),
// getContactsForces, updateAngular, updateRotationMatrix, updateVertices).
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles it with the reference's sources into
// oracle/_ref/ (serially in libdelta_ref.so, with OpenMP in libdelta_ref_omp.so, the timed
// CPU baseline of the time step).  It includes no header that carries the ICC-only
// `nomask` clause (penalty.h:119), so it builds under GCC's OpenMP.
#include <algorithm>
#include <cstdint>
#include <utility>
#include <vector>

#include "contact/contactpoint.h"
#include "contact/detection/bf.h"
#include "contact/forces/forces.h"
#include "dynamics/dynamics.h"

namespace det = delta::contact::detection;

extern "C" {

// ---- a whole time step with the reference's functions ------------------------------------
// The update order of the oracle's dor_sim_run (multiscale Collision.cpp / MoveParticles.cpp):
// forces from the previous detection's contacts (getContactsForces per partner, partners
// in ascending order, the slave side with the inverted normal), v += dt F/m and
// updateAngular for the bodies with contacts, then v += dt g, x += dt v,
// updateRotationMatrix and updateVertices for every moving body, then detection: candidate
// pairs i < j (not both obstacles) whose bounding spheres grown by the epsilons overlap,
// each run through the reference's bf() over all of its triangle pairs.  The body and
// triangle arrays are dor_scene's (delta_oracle.h).  getContactsForces uses the constants
// compiled into forces.cpp (SPRING 1e4, DAMPER 0.5, FRICTION 0.5).  Candidate pairs and
// bodies are spread over the threads with OpenMP (both builds); each bf() call and each
// body's sum over its partners runs serially, so the result does not depend on the
// threads.
struct ref_scene {
  int32_t n_bodies;
  const int64_t *tri_offset;
  double *x, *y, *z;
  const double *rx, *ry, *rz;
  double *pos;
  const double *ref_pos;
  double *vel, *ang, *ref_ang, *rot;
  const double *inertia, *inverse, *mass, *eps, *radius;
  const uint8_t *friction, *obstacle;
};

struct ref_sim {
  std::vector<std::pair<int32_t, int32_t>> pairs;                  // candidate pairs of the last detection
  std::vector<std::vector<delta::contact::contactpoint>> contacts;  // per pair, A = first
};

ref_sim *ref_sim_create() { return new ref_sim(); }
void ref_sim_destroy(ref_sim *s) { delete s; }

static void ref_sim_detect(ref_sim *s, const ref_scene *sc) {
  const int32_t nb = sc->n_bodies;
  std::vector<std::vector<std::pair<int32_t, int32_t>>> per(nb);
#pragma omp parallel for schedule(dynamic, 16)
  for (int32_t i = 0; i < nb; ++i)
    for (int32_t j = i + 1; j < nb; ++j) {
      if (sc->obstacle[i] && sc->obstacle[j]) continue;
      const double dx = sc->pos[3 * j] - sc->pos[3 * i], dy = sc->pos[3 * j + 1] - sc->pos[3 * i + 1],
                   dz = sc->pos[3 * j + 2] - sc->pos[3 * i + 2];
      const double reach = sc->radius[i] + sc->radius[j] + sc->eps[i] + sc->eps[j];
      if (dx * dx + dy * dy + dz * dz > reach * reach * (1.0 + 1e-9) + 1e-18) continue;
      per[i].push_back({i, j});
    }
  s->pairs.clear();
  for (auto &v : per) s->pairs.insert(s->pairs.end(), v.begin(), v.end());
  s->contacts.assign(s->pairs.size(), {});
  const int64_t np = (int64_t)s->pairs.size();
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t k = 0; k < np; ++k) {
    const int32_t i = s->pairs[k].first, j = s->pairs[k].second;
    const int64_t a0 = sc->tri_offset[i], b0 = sc->tri_offset[j];
    s->contacts[k] = det::bf(sc->x + 3 * a0, sc->y + 3 * a0, sc->z + 3 * a0, (int)(sc->tri_offset[i + 1] - a0),
                             sc->eps[i], sc->friction[i] != 0, i, sc->x + 3 * b0, sc->y + 3 * b0, sc->z + 3 * b0,
                             (int)(sc->tri_offset[j + 1] - b0), sc->eps[j], sc->friction[j] != 0, j);
  }
}

// Runs nsteps; returns the contact count of the last detection.
int64_t ref_sim_run(ref_sim *s, ref_scene *sc, double dt, const double gravity[3], int32_t nsteps,
                    int64_t *contacts_per_step) {
  const int32_t nb = sc->n_bodies;
  std::vector<double> F(3 * (size_t)nb), T(3 * (size_t)nb);
  std::vector<uint8_t> has((size_t)nb);
  for (int32_t step = 0; step < nsteps; ++step) {
    // partners of every body, ascending, with the index of the pair's contact list
    std::vector<std::vector<std::pair<int32_t, int64_t>>> partners(nb);
    for (int64_t k = 0; k < (int64_t)s->pairs.size(); ++k) {
      if (s->contacts[k].empty()) continue;
      partners[s->pairs[k].first].push_back({s->pairs[k].second, k});
      partners[s->pairs[k].second].push_back({s->pairs[k].first, k});
    }
#pragma omp parallel for schedule(dynamic, 16)
    for (int32_t i = 0; i < nb; ++i) {
      double *Fi = &F[3 * (size_t)i], *Ti = &T[3 * (size_t)i];
      Fi[0] = Fi[1] = Fi[2] = Ti[0] = Ti[1] = Ti[2] = 0.0;
      has[i] = 0;
      if (sc->obstacle[i]) continue;
      auto &pl = partners[i];
      std::sort(pl.begin(), pl.end());
      for (const auto &pk : pl) {
        const int32_t j = pk.first;
        std::vector<delta::contact::contactpoint> c = s->contacts[pk.second];
        if (i > j)
          for (auto &cp : c)
            for (int d = 0; d < 3; ++d) cp.normal[d] = -1.0 * cp.normal[d];
        double rf[3] = {0, 0, 0}, rt[3] = {0, 0, 0}, pi[3], pj[3], rpi[3], rpj[3], ai[3], aj[3], rai[3], raj[3],
               li[3], lj[3], Ii[9], Ij[9], Ri[9], Rj[9];
        for (int d = 0; d < 3; ++d) {
          pi[d] = sc->pos[3 * i + d], pj[d] = sc->pos[3 * j + d];
          rpi[d] = sc->ref_pos[3 * i + d], rpj[d] = sc->ref_pos[3 * j + d];
          ai[d] = sc->ang[3 * i + d], aj[d] = sc->ang[3 * j + d];
          rai[d] = sc->ref_ang[3 * i + d], raj[d] = sc->ref_ang[3 * j + d];
          li[d] = sc->vel[3 * i + d], lj[d] = sc->vel[3 * j + d];
        }
        for (int d = 0; d < 9; ++d) {
          Ii[d] = sc->inverse[9 * i + d], Ij[d] = sc->inverse[9 * j + d];
          Ri[d] = sc->rot[9 * i + d], Rj[d] = sc->rot[9 * j + d];
        }
        delta::contact::forces::getContactsForces(c, pi, rpi, ai, rai, li, sc->mass[i], Ii, Ri, 0, pj, rpj, aj, raj,
                                                  lj, sc->mass[j], Ij, Rj, 0, rf, rt, false);
        for (int d = 0; d < 3; ++d) Fi[d] += rf[d], Ti[d] += rt[d];
        has[i] = 1;
      }
    }
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < nb; ++i) {
      if (has[i]) {
        for (int d = 0; d < 3; ++d) sc->vel[3 * i + d] += dt * (F[3 * (size_t)i + d] / sc->mass[i]);
        delta::dynamics::updateAngular(sc->ref_ang + 3 * i, sc->rot + 9 * i, const_cast<double *>(sc->inertia) + 9 * i,
                                       const_cast<double *>(sc->inverse) + 9 * i, &T[3 * (size_t)i], dt);
      }
      if (sc->obstacle[i]) continue;
      for (int d = 0; d < 3; ++d) sc->vel[3 * i + d] += dt * (gravity[d]);
      for (int d = 0; d < 3; ++d) sc->pos[3 * i + d] += dt * sc->vel[3 * i + d];
      delta::dynamics::updateRotationMatrix(sc->ang + 3 * i, sc->ref_ang + 3 * i, sc->rot + 9 * i, dt);
      for (int64_t v = 3 * sc->tri_offset[i]; v < 3 * sc->tri_offset[i + 1]; ++v)
        delta::dynamics::updateVertices(&sc->x[v], &sc->y[v], &sc->z[v], const_cast<double *>(sc->rx) + v,
                                        const_cast<double *>(sc->ry) + v, const_cast<double *>(sc->rz) + v,
                                        sc->rot + 9 * i, sc->pos + 3 * i, const_cast<double *>(sc->ref_pos) + 3 * i);
    }
    ref_sim_detect(s, sc);
    int64_t nc = 0;
    for (const auto &c : s->contacts) nc += (int64_t)c.size();
    if (contacts_per_step) contacts_per_step[step] = nc;
  }
  int64_t nc = 0;
  for (const auto &c : s->contacts) nc += (int64_t)c.size();
  return nc;
}

}  // extern "C"
