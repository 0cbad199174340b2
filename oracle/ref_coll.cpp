/* Host build of the reference collision module (collision_kernels9/kernel.cu
 * and the headers it includes), read in place through ref_shim/shim.h.
 * TEST INFRASTRUCTURE ONLY (oracle/_ref).
 *
 * Entry points:
 *   ref_pt                   -> pt, point_triange_v2.h:589-841
 *   ref_dtn                  -> dtn, dist_node2tri.h:14-129
 *   ref_narrow_phase_kernel  -> kNarrowPhase_new, narrowphase.h:46-155
 *   ref_closest_face_kernel  -> kFindClosestFace, narrowphase.h:159-201
 *   ref_collision_kernel     -> kCollisionResponseForce, collision_response.h:38-127
 */
#include "shim.h"
#include <omp.h>

namespace icf_ref_coll {
#include "kernel.cu"
}

extern "C" {

/* x[12] = (p, v0, v1, v2); fd[12], sd[144] written (zero-filled first, as
 * the caller in collision_response.h:71-72 does). Returns the squared
 * distance. */
double ref_pt(const double *x, double *fd, double *sd, double *s, double *t,
              int *branch) {
  double lx[12], lfd[12] = {}, lsd[12][12] = {};
  for (int i = 0; i < 12; i++) lx[i] = x[i];
  double os = 0, ot = 0;
  int br = -1;
  double d = icf_ref_coll::pt(lx, lfd, lsd, os, ot, br);
  for (int i = 0; i < 12; i++) fd[i] = lfd[i];
  std::memcpy(sd, lsd, sizeof(lsd));
  *s = os;
  *t = ot;
  *branch = br;
  return d;
}

/* f[9] = triangle vertices, p[3] = point. */
double ref_dtn(const double *f, const double *p) {
  return icf_ref_coll::dtn(f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7],
                           f[8], p[0], p[1], p[2]);
}

void ref_narrow_phase_kernel(int nPairs, const double *dn, const int *ie,
                             int *narrowList, int el_all_stride,
                             int nd_stride, int nthreads) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nPairs; i++) {
    icf_shim_set_thread(i);
    icf_ref_coll::kNarrowPhase_new(nPairs, dn, ie, narrowList, el_all_stride,
                                   nd_stride);
  }
}

void ref_closest_face_kernel(int nPairs, int tet_stride, int *narrowList2,
                             const double *dn, const int *ie,
                             const int *faces, int nd_stride,
                             int el_all_stride, int fc_stride, int nthreads) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nPairs; i++) {
    icf_shim_set_thread(i);
    icf_ref_coll::kFindClosestFace(nPairs, tet_stride, narrowList2, dn, ie,
                                   faces, nd_stride, el_all_stride, fc_stride);
  }
}

void ref_collision_kernel(const int *icr, double *dn, double h, double *vals,
                          double *rhs, int nImpacts, int cr_stride,
                          int nd_stride, double k, double distanceEpsilon,
                          int nthreads) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nImpacts; i++) {
    icf_shim_set_thread(i);
    icf_ref_coll::kCollisionResponseForce(icr, dn, h, vals, rhs, nImpacts,
                                          cr_stride, nd_stride, k,
                                          distanceEpsilon);
  }
}

}  // extern "C"
