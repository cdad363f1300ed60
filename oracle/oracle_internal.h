/*
 * oracle_internal.h -- helpers shared by the oracle's translation units (test
 * infrastructure only; see delta_oracle.h).
 */
#ifndef DELTA_ORACLE_INTERNAL_H
#define DELTA_ORACLE_INTERNAL_H

/* One edge-edge feature of bfSolver (bf.cpp:586-697): Sunday's clamped parameters of
 * the edges HA<-TA and HB<-TB and the distance of the resulting point pair. */
double dor_seg_seg_feature(const double *HA, const double *TA, const double *HB, const double *TB,
                           double *sc_out, double *tc_out);
/* One vertex-face feature of bfSolver (bf.cpp:920-1090): X against (V0,V1,V2). */
double dor_pt_tri_feature(const double *V0, const double *V1, const double *V2, const double *X,
                          double *s_out, double *t_out);

#endif
