// icf_tet.cuh -- the per-tetrahedron arithmetic of the assembly, shared by the
// tet kernel (k_tet_unit, which stages the results) and the fused row-tile
// kernel (k_tile_fused, which keeps them in shared memory): both evaluate the
// same code, so their records are bit-identical.
//
// F_and_Df_Corotational and kelElementElasticityForce
// (elem_kernels9/element_kernels2.h:19-159, :195-263) in closed form.
#pragma once
#include <cuda_runtime.h>

#include "icf_internal.cuh"

// ---- small vector helpers ---------------------------------------------------
// A node position (32 B, 32 B aligned: node arrays start on 256 B) in one
// 256-bit read-only load.
static __device__ __forceinline__ void ld_node(const double4 *__restrict__ p, int i,
                                        double o[3]) {
  double w;
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
      : "=d"(o[0]), "=d"(o[1]), "=d"(o[2]), "=d"(w)
      : "l"(p + i));
  asm("" ::"d"(w));  // the fourth component is padding
}

// Orthonormal frame of three points as in fastRotationMatrix
// (elem_kernels9/matrix_math1.h:32-71): columns unit(p1-p0),
// unit((p1-p0) x (p2-p0)), unit(col1 x col0).
static __device__ __forceinline__ void frame3(const double p0[3], const double p1[3],
                                       const double p2[3], double R[3][3]) {
  double d[3], w[3];
  for (int k = 0; k < 3; k++) {
    d[k] = p1[k] - p0[k];
    w[k] = p2[k] - p0[k];
  }
  double r = rsqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  for (int k = 0; k < 3; k++) R[k][0] = d[k] * r;
  double c0 = -d[2] * w[1] + d[1] * w[2];
  double c1 = d[2] * w[0] - d[0] * w[2];
  double c2 = -d[1] * w[0] + d[0] * w[1];
  r = rsqrt(c0 * c0 + c1 * c1 + c2 * c2);
  R[0][1] = c0 * r;
  R[1][1] = c1 * r;
  R[2][1] = c2 * r;
  c0 = R[1][1] * R[2][0] - R[1][0] * R[2][1];
  c1 = -R[0][1] * R[2][0] + R[0][0] * R[2][1];
  c2 = R[0][1] * R[1][0] - R[0][0] * R[1][1];
  r = rsqrt(c0 * c0 + c1 * c1 + c2 * c2);
  R[0][2] = c0 * r;
  R[1][2] = c1 * r;
  R[2][2] = c2 * r;
}

// ---- tetrahedra ---------------------------------------------------------------
// Closed form of the reference's K = V B^T E B for isotropic E:
//   K_ab = V (lam g_a g_b^T + mu g_b g_a^T + mu (g_a.g_b) I)
// so that, with h_b = R g_b (R = R1 R0^T, the corotational rotation),
//   Df_ab = R K_ab R^T = V (lam h_a h_b^T + mu h_b h_a^T + mu (h_a.h_b) I)
//   f_a   = R sum_b K_ab xr_b = V R sigma(F) g_a,  F = sum_b xr_b g_b^T,
//           sigma(F) = lam tr(F) I + mu (F + F^T),  xr_b = R^T xc_b - x0_b
//   sum_b Df_ab v_b = V (lam tr(L) I + mu (L + L^T)) h_a,  L = sum_b v_b h_b^T
// and the consistent mass is M_ab = rho/20 (1 + delta_ab) I.  The staging
// record of vertex a is {h_a, V} and {rhs_a, 0}; k_gather rebuilds
// LHS_ab = stiffCoeff Df_ab + massCoeff M_ab from it.  The record (16
// double2, 256 B) is written to rec in shared memory.
// The outputs of one tet: rotated gradients h_a, rest volume V, and the
// Newmark rhs of each vertex.
struct icf_tet_out {
  double h[4][3];
  double V;
  double r[4][3];
};

static __device__ __forceinline__ void tet_eval(int e, const int4 *__restrict__ elem,
                                                const double4 *__restrict__ x0,
                                                const double4 *__restrict__ xc,
                                                const double2 *__restrict__ va, const icf_dprm &P,
                                                icf_tet_out &o) {
  const int4 id = __ldg(elem + e);
  const int nid[4] = {id.x, id.y, id.z, id.w};
  double X[4][3], C[4][3], Vn[4][3], An[4][3];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    ld_node(x0, nid[i], X[i]);
    ld_node(xc, nid[i], C[i]);
    const double2 q0 = __ldg(va + 3 * nid[i]), q1 = __ldg(va + 3 * nid[i] + 1),
                  q2 = __ldg(va + 3 * nid[i] + 2);
    Vn[i][0] = q0.x; Vn[i][1] = q0.y; Vn[i][2] = q1.x;
    An[i][0] = q1.y; An[i][1] = q2.x; An[i][2] = q2.y;
  }
  // rest volume and shape-function gradients (element_kernels2.h:38-57)
  const double x12 = X[0][0] - X[1][0], x13 = X[0][0] - X[2][0], x14 = X[0][0] - X[3][0];
  const double x23 = X[1][0] - X[2][0], x24 = X[1][0] - X[3][0], x34 = X[2][0] - X[3][0];
  const double y12 = X[0][1] - X[1][1], y13 = X[0][1] - X[2][1], y14 = X[0][1] - X[3][1];
  const double y23 = X[1][1] - X[2][1], y24 = X[1][1] - X[3][1], y34 = X[2][1] - X[3][1];
  const double z12 = X[0][2] - X[1][2], z13 = X[0][2] - X[2][2], z14 = X[0][2] - X[3][2];
  const double z23 = X[1][2] - X[2][2], z24 = X[1][2] - X[3][2], z34 = X[2][2] - X[3][2];
  const double Jdet = -x12 * (y23 * z34 - y34 * z23) - x23 * (y34 * z12 - y12 * z34) -
                      x34 * (y12 * z23 - y23 * z12);
  const double V = Jdet / 6.;
  const double iJ = 1.0 / Jdet;
  double g[4][3];
  g[0][0] = (y24 * z23 - y23 * z24) * iJ;  // a1 = y42 z32 - y32 z42
  g[0][1] = (x23 * z24 - x24 * z23) * iJ;  // b1 = x32 z42 - x42 z32
  g[0][2] = (x24 * y23 - x23 * y24) * iJ;  // c1 = x42 y32 - x32 y42
  g[1][0] = (y13 * z34 - y34 * z13) * iJ;  // a2 = y31 z43 - y34 z13
  g[1][1] = (x34 * z13 - x13 * z34) * iJ;  // b2 = x43 z31 - x13 z34
  g[1][2] = (x13 * y34 - x34 * y13) * iJ;  // c2 = x31 y43 - x34 y13
  g[2][0] = (y24 * z14 - y14 * z24) * iJ;  // a3
  g[2][1] = (x14 * z24 - x24 * z14) * iJ;  // b3
  g[2][2] = (x24 * y14 - x14 * y24) * iJ;  // c3
  g[3][0] = (y12 * z13 - y13 * z12) * iJ;  // a4 = y13 z21 - y12 z31
  g[3][1] = (x13 * z12 - x12 * z13) * iJ;  // b4 = x21 z13 - x31 z12
  g[3][2] = (x12 * y13 - x13 * y12) * iJ;  // c4 = x13 y21 - x12 y31

  // corotational rotation R = R1 R0^T (:175-201)
  double R0[3][3], R1[3][3], R[3][3];
  frame3(X[0], X[1], X[2], R0);
  frame3(C[0], C[1], C[2], R1);
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
      R[i][j] = R1[i][0] * R0[j][0] + R1[i][1] * R0[j][1] + R1[i][2] * R0[j][2];

  // F = sum_b (R^T xc_b - x0_b) g_b^T and the stress sigma(F)
  double F[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
  for (int b = 0; b < 4; b++) {
    double xr[3];
#pragma unroll
    for (int k = 0; k < 3; k++)
      xr[k] = (C[b][0] * R[0][k] + C[b][1] * R[1][k] + C[b][2] * R[2][k]) - X[b][k];
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
      for (int l = 0; l < 3; l++) F[k][l] += xr[k] * g[b][l];
  }
  const double trF = F[0][0] + F[1][1] + F[2][2];
  double S[3][3];
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int l = 0; l < 3; l++)
      S[k][l] = P.mu * (F[k][l] + F[l][k]) + (k == l ? P.lam * trF : 0.0);

  // rotated gradients h_b = R g_b and L = sum_b v_b h_b^T
  double h[4][3];
  double L[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  double sv[3] = {0, 0, 0}, sa[3] = {0, 0, 0};
#pragma unroll
  for (int b = 0; b < 4; b++) {
#pragma unroll
    for (int k = 0; k < 3; k++)
      h[b][k] = R[k][0] * g[b][0] + R[k][1] * g[b][1] + R[k][2] * g[b][2];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      sv[k] += Vn[b][k];
      sa[k] += An[b][k];
#pragma unroll
      for (int l = 0; l < 3; l++) L[k][l] += Vn[b][k] * h[b][l];
    }
  }
  const double trL = L[0][0] + L[1][1] + L[2][2];
  const double mV = P.rho20 * V;
  const double gz = P.grav_rho * V / 4;

#pragma unroll
  for (int a = 0; a < 4; a++) {
    double sg[3], f[3], dv[3], r[3];
#pragma unroll
    for (int k = 0; k < 3; k++) sg[k] = S[k][0] * g[a][0] + S[k][1] * g[a][1] + S[k][2] * g[a][2];
#pragma unroll
    for (int k = 0; k < 3; k++) f[k] = V * (R[k][0] * sg[0] + R[k][1] * sg[1] + R[k][2] * sg[2]);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const double Lh = (L[k][0] + L[0][k]) * h[a][0] + (L[k][1] + L[1][k]) * h[a][1] +
                        (L[k][2] + L[2][k]) * h[a][2];
      dv[k] = V * (P.lam * trL * h[a][k] + P.mu * Lh);
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const double damp = mV * P.dm * (Vn[a][k] + sv[k]) + P.ds * dv[k];
      const double inert = mV * (An[a][k] + sa[k]);
      r[k] = (k == 2 ? gz : 0.0) - f[k] - damp - inert;
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
      o.h[a][k] = h[a][k];
      o.r[a][k] = r[k];
    }
  }
  o.V = V;
}

// The staging record of one tet (16 double2, 256 B).  FP64: {h_a, V} for
// a = 0..3, then {rhs_a, 0}.  FP32-mixed: {rhs_a, 0} (FP64) for a = 0..3, then
// the FP32 {h_a, V} as four float4 (the Hessian inputs rounded to FP32).
template <bool MIXED>
static __device__ __forceinline__ void tet_record(int e, const int4 *__restrict__ elem,
                                                  const double4 *__restrict__ x0,
                                                  const double4 *__restrict__ xc,
                                                  const double2 *__restrict__ va, const icf_dprm &P,
                                                  double2 *rec) {
  icf_tet_out o;
  tet_eval(e, elem, x0, xc, va, P, o);
#pragma unroll
  for (int a = 0; a < 4; a++) {
    if (MIXED) {
      rec[2 * a] = make_double2(o.r[a][0], o.r[a][1]);
      rec[2 * a + 1] = make_double2(o.r[a][2], 0.0);
      *reinterpret_cast<float4 *>(rec + 8 + a) =
          make_float4((float)o.h[a][0], (float)o.h[a][1], (float)o.h[a][2], (float)o.V);
    } else {
      rec[2 * a] = make_double2(o.h[a][0], o.h[a][1]);
      rec[2 * a + 1] = make_double2(o.h[a][2], o.V);
      rec[8 + 2 * a] = make_double2(o.r[a][0], o.r[a][1]);
      rec[9 + 2 * a] = make_double2(o.r[a][2], 0.0);
    }
  }
}

