// icf_collide.cuh -- the narrow-phase point-in-tet test and the broad phase's
// pair rule, shared by the pair pipeline (icf_broad.cu k_pairs, icf_contact.cu
// k_narrow) and the direct contact detection (icf_broad.cu k_detect).
//
// Every file that includes this header is compiled with -fmad=false, so the
// inverse and the barycentric test round every product and sum on its own, in
// the order written, and give the same bits wherever they are evaluated.
#pragma once

#include "icf_internal.cuh"

// Inverse of the edge matrix [x1 - x0, x2 - x0, x3 - x0] of a tet, in the
// reference's expression order (kNarrowPhase_new, narrowphase.h:3-44).
static __device__ __forceinline__ void tet_inverse(const double *x, double b[9]) {
  const double a11 = x[3] - x[0], a12 = x[6] - x[0], a13 = x[9] - x[0];
  const double a21 = x[4] - x[1], a22 = x[7] - x[1], a23 = x[10] - x[1];
  const double a31 = x[5] - x[2], a32 = x[8] - x[2], a33 = x[11] - x[2];
  const double det = a31 * (-a13 * a22 + a12 * a23) + a32 * (a13 * a21 - a11 * a23) +
                     a33 * (-a12 * a21 + a11 * a22);
  b[0] = (-a23 * a32 + a22 * a33) / det;
  b[1] = (a13 * a32 - a12 * a33) / det;
  b[2] = (-a13 * a22 + a12 * a23) / det;
  b[3] = (a23 * a31 - a21 * a33) / det;
  b[4] = (-a13 * a31 + a11 * a33) / det;
  b[5] = (a13 * a21 - a11 * a23) / det;
  b[6] = (-a22 * a31 + a21 * a32) / det;
  b[7] = (a12 * a31 - a11 * a32) / det;
  b[8] = (-a12 * a21 + a11 * a22) / det;
}

// (x, y, z) relative to the tet's first vertex strictly inside it, with the
// reference's 1e-10 margin on the barycentric coordinates (narrowphase.h:20-44).
static __device__ __forceinline__ bool tet_contains(const double b[9], double x, double y, double z) {
  const double eps = 1E-10;
  const double y1 = x * b[0] + y * b[1] + z * b[2];
  const double y2 = x * b[3] + y * b[4] + z * b[5];
  const double y3 = x * b[6] + y * b[7] + z * b[8];
  return (y1 > eps && y2 > eps && y3 > eps && (y1 + y2 + y3) < (1 - eps));
}

// A vertex of one element inside the other's box (closed); lh = {lo[3], hi[3]}.
static __device__ __forceinline__ bool vertex_in_box(const int n[4], const double4 *xc, const double *lh) {
#pragma unroll
  for (int v = 0; v < 4; v++) {
    const double4 p = xc[n[v]];
    if (p.x >= lh[0] && p.x <= lh[3] && p.y >= lh[1] && p.y <= lh[4] && p.z >= lh[2] && p.z <= lh[5])
      return true;
  }
  return false;
}

// The broad phase's pair rule for surface elements a and b (symmetric):
// boxes overlap, no node in common (the narrow phase skips such pairs,
// kNarrowPhase_new, narrowphase.h:67-70), a vertex of one inside the other's
// box (an impact needs a vertex inside the other tet, so this drops no pair
// that can give one), and different groups when groups are set.
static __device__ __forceinline__ bool keep_pair(int a, int b, const double *lohi, const int *group,
                                                 const int4 *selem, const double4 *xc) {
  if (group && group[a] == group[b]) return false;
  for (int k = 0; k < 3; k++)
    if (!(lohi[6 * (size_t)a + k] <= lohi[6 * (size_t)b + 3 + k] && lohi[6 * (size_t)b + k] <= lohi[6 * (size_t)a + 3 + k]))
      return false;
  const int4 p = selem[a], q = selem[b];
  const int pa[4] = {p.x, p.y, p.z, p.w}, qb[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
      if (pa[i] == qb[j]) return false;
  return vertex_in_box(pa, xc, lohi + 6 * (size_t)b) || vertex_in_box(qb, xc, lohi + 6 * (size_t)a);
}
