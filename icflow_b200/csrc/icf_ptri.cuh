// icf_ptri.cuh -- the Voronoi region of the point-triangle distance.
//
// The region of pt (point_triange_v2.h:589-841), its barycentric coordinates
// (s, t) and the squared distance, evaluated exactly as the CPU checker does.
// Every file that includes this header is compiled with -fmad=false, so each
// product and sum rounds on its own, in the order written, and the region (an
// integer outcome of floating-point comparisons) is the same bit for bit.
#pragma once

#include "icf_internal.cuh"

namespace {

// The Voronoi region of pt (point_triange_v2.h:589-841), its barycentric
// coordinates (s, t) and the squared distance, evaluated exactly as the CPU
// checker does.  The derivatives are computed separately (icf_contact_deriv.cu)
// once the region is known.  x = (p, v0, v1, v2); kind 0 = interior (plane),
// 1 = vertex (block ib), 2 = edge (blocks ia, ib, nearer endpoint first).
struct pt_cls {
  int kind, ia, ib;
  double s, t, dsq;
};

__device__ double vv_dsq(const double x[12], int ia, int ib) {
  double dsq = 0;
  for (int k = 0; k < 3; k++) {
    const double d = x[3 * ia + k] - x[3 * ib + k];
    dsq += d * d;
  }
  return dsq;
}

// distance to the line through the edge, nearer endpoint first
// (vertex_edge_distance_and_derivs_12, :237-294, and :152-177)
__device__ double ve_dsq(const double x[12], int &ia, int &ib) {
  double da = 0, db = 0;
  for (int k = 0; k < 3; k++) {
    da += (x[k] - x[3 * ia + k]) * (x[k] - x[3 * ia + k]);
    db += (x[k] - x[3 * ib + k]) * (x[k] - x[3 * ib + k]);
  }
  if (da > db) {
    const int s = ia;
    ia = ib;
    ib = s;
  }
  const double *P = x, *Q1 = x + 3 * ia, *Q2 = x + 3 * ib;
  double el2 = 0, rde = 0;
  for (int k = 0; k < 3; k++) {
    el2 += (Q2[k] - Q1[k]) * (Q2[k] - Q1[k]);
    rde += (Q1[k] - P[k]) * (Q2[k] - Q1[k]);
  }
  const double t = -rde / el2, u = 1 - t;
  double dist2 = 0;
  for (int k = 0; k < 3; k++) {
    const double d = P[k] - u * Q1[k] - t * Q2[k];
    dist2 += d * d;
  }
  return dist2;
}

// squared distance to the plane through the barycentric foot point
// (point_plane_distance, :449-492)
__device__ double plane_dsq(const double x[12]) {
  const double *P = x, *V0 = x + 3, *V1 = x + 6, *V2 = x + 9;
  double e0[3], e1[3], w[3];
  for (int k = 0; k < 3; k++) {
    e0[k] = -V0[k] + V1[k];
    e1[k] = -V0[k] + V2[k];
    w[k] = -P[k] + V0[k];
  }
  const double a = e0[0] * e0[0] + e0[1] * e0[1] + e0[2] * e0[2];
  const double b = e1[1] * e0[1] + e1[2] * e0[2] + e0[0] * e1[0];
  const double c = e1[1] * e1[1] + e1[2] * e1[2] + e1[0] * e1[0];
  const double d = w[0] * e0[0] + w[1] * e0[1] + w[2] * e0[2];
  const double e = e1[1] * w[1] + e1[2] * w[2] + w[0] * e1[0];
  const double det = a * c - b * b;
  const double inv = 1. / det;
  const double s = (b * e - c * d) * inv, t = (b * d - a * e) * inv;
  const double u = 1 - (s + t);
  double dist2 = 0;
  for (int k = 0; k < 3; k++) {
    const double q = -P[k] + V1[k] * s + V2[k] * t + V0[k] * u;
    dist2 += q * q;
  }
  return dist2;
}

__device__ pt_cls pt_classify(const double x[12]) {
  pt_cls r;
  r.ia = r.ib = 0;
  const double *P = x, *V0 = x + 3, *V1 = x + 6, *V2 = x + 9;
  double e0[3], e1[3], w[3];
  for (int k = 0; k < 3; k++) {
    e0[k] = -V0[k] + V1[k];
    e1[k] = -V0[k] + V2[k];
    w[k] = -P[k] + V0[k];
  }
  const double a = e0[0] * e0[0] + e0[1] * e0[1] + e0[2] * e0[2];
  const double b = e1[1] * e0[1] + e1[2] * e0[2] + e0[0] * e1[0];
  const double c = e1[1] * e1[1] + e1[2] * e1[2] + e1[0] * e1[0];
  const double d = w[0] * e0[0] + w[1] * e0[1] + w[2] * e0[2];
  const double e = e1[1] * w[1] + e1[2] * w[2] + w[0] * e1[0];
  const double det = a * c - b * b;
  double s = b * e - c * d, t = b * d - a * e;
  // vertex / edge selectors: vertex k = block k; edge (i, j) as passed by pt
#define VV(k) do { r.kind = 1; r.ib = (k); r.dsq = vv_dsq(x, 0, (k)); } while (0)
#define VE(i, j) do { r.kind = 2; r.ia = (i); r.ib = (j); r.dsq = ve_dsq(x, r.ia, r.ib); } while (0)
  if (s + t <= det) {
    if (s < 0) {
      if (t < 0 && d < 0) {
        t = 0;
        if (-d >= a) { s = 1; VV(2); }
        else { s = -d / a; VE(2, 1); }
      } else {
        s = 0;
        if (e >= 0) { t = 0; VV(1); }
        else if (-e >= c) { t = 1; VV(3); }
        else { t = -e / c; VE(3, 1); }
      }
    } else if (t < 0) {
      t = 0;
      if (d >= 0) { s = 0; VV(1); }
      else if (-d >= a) { s = 1; VV(2); }
      else { s = -d / a; VE(1, 2); }
    } else {
      const double inv = (1) / det;
      s *= inv;
      t *= inv;
      r.kind = 0;
      r.dsq = plane_dsq(x);
    }
  } else {
    if (s < 0) {
      const double t0 = b + d, t1 = c + e;
      if (t1 > t0) {
        const double num = t1 - t0, den = a - 2 * b + c;
        if (num >= den) { s = 1; t = 0; VV(2); }
        else { s = num / den; t = 1 - s; VE(2, 3); }
      } else {
        s = 0;
        if (t1 <= 0) { t = 1; VV(3); }
        else if (e >= 0) { t = 0; VV(1); }
        else { t = -e / c; VE(1, 3); }
      }
    } else if (t < 0) {
      const double t0 = b + e, t1 = a + d;
      if (t1 > t0) {
        const double num = t1 - t0, den = a - 2 * b + c;
        if (num >= den) { t = 1; s = 0; VV(3); }
        else { t = num / den; s = 1 - t; VE(2, 3); }
      } else {
        t = 0;
        if (t1 <= 0) { s = 1; VV(2); }
        else if (d >= 0) { s = 0; VV(1); }
        else { s = -d / a; VE(1, 2); }
      }
    } else {
      const double num = c + e - b - d;
      if (num <= 0) { s = 0; t = 1; VV(3); }
      else {
        const double den = a - 2 * b + c;
        if (num >= den) { s = 1; t = 0; VV(2); }
        else { s = num / den; t = 1 - s; VE(2, 3); }
      }
    }
  }
#undef VV
#undef VE
  r.s = s;
  r.t = t;
  return r;
}

}  // namespace
