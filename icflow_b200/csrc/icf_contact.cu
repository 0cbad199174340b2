// icf_contact.cu -- narrow phase, closest face and penalty contact.
//
// This file is compiled with -fmad=false: every product and sum is rounded on
// its own, in the order written, so the integer outputs that hinge on
// floating-point comparisons (the 8-bit inclusion masks, the closest face,
// the Voronoi region of the point-triangle distance) are reproducible bit for
// bit against a CPU evaluation with the same operation order.
//
//   k_narrow      kNarrowPhase_new (collision_kernels9/narrowphase.h:46-155)
//   k_expand      the host set expansion of GPU_Functionality.cs:566-580,
//                 done on the device as keys (node << 32 | element)
//   k_closest     kFindClosestFace (narrowphase.h:159-201) with dtn
//                 (dist_node2tri.h:14-129)
//   k_imp_unit    kCollisionResponseForce (collision_response.h:38-127) with
//                 the point-triangle distance derivatives pt()
//                 (point_triange_v2.h:13-841)
#include <cub/cub.cuh>

#include "icf_internal.cuh"

namespace {

// ---- narrow phase ---------------------------------------------------------------
__device__ void tet_inverse(const double *x, double b[9]) {
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

__device__ bool tet_contains(const double b[9], double x, double y, double z) {
  const double eps = 1E-10;
  const double y1 = x * b[0] + y * b[1] + z * b[2];
  const double y2 = x * b[3] + y * b[4] + z * b[5];
  const double y3 = x * b[6] + y * b[7] + z * b[8];
  return (y1 > eps && y2 > eps && y3 > eps && (y1 + y2 + y3) < (1 - eps));
}

__global__ void k_narrow(int np, const int *__restrict__ pairs,
                         const int4 *__restrict__ selem,
                         const double4 *__restrict__ xc, int *__restrict__ masks,
                         int *__restrict__ counts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const int4 A = selem[pairs[2 * i]], B = selem[pairs[2 * i + 1]];
  const int na[4] = {A.x, A.y, A.z, A.w}, nb[4] = {B.x, B.y, B.z, B.w};
  int m = 0;
  bool shared = false;
  for (int p = 0; p < 4; p++)
    for (int q = 0; q < 4; q++) shared |= (na[p] == nb[q]);
  if (!shared) {
    double xa[12], xb[12];
    for (int k = 0; k < 4; k++) {
      const double4 pa = xc[na[k]], pb = xc[nb[k]];
      xa[3 * k] = pa.x; xa[3 * k + 1] = pa.y; xa[3 * k + 2] = pa.z;
      xb[3 * k] = pb.x; xb[3 * k + 1] = pb.y; xb[3 * k + 2] = pb.z;
    }
    double ba[9], bb[9];
    tet_inverse(xa, ba);
    tet_inverse(xb, bb);
    for (int k = 0; k < 4; k++)
      if (tet_contains(ba, xb[3 * k] - xa[0], xb[3 * k + 1] - xa[1], xb[3 * k + 2] - xa[2]))
        m |= 1 << k;
    for (int k = 0; k < 4; k++)
      if (tet_contains(bb, xa[3 * k] - xb[0], xa[3 * k + 1] - xb[1], xa[3 * k + 2] - xb[2]))
        m |= 16 << k;
  }
  masks[i] = m;
  counts[i] = __popc(m);
}

// (node << 32 | element) for every set bit; bit k < 4: vertex k of the second
// element is inside the first; bit 4+k: vertex k of the first inside the second.
__global__ void k_expand(int np, const int *__restrict__ pairs,
                         const int4 *__restrict__ selem, const int *__restrict__ masks,
                         const int *__restrict__ off,
                         unsigned long long *__restrict__ keys) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const int m = masks[i];
  if (!m) return;
  const int ea = pairs[2 * i], eb = pairs[2 * i + 1];
  const int4 A = selem[ea], B = selem[eb];
  const int na[4] = {A.x, A.y, A.z, A.w}, nb[4] = {B.x, B.y, B.z, B.w};
  int w = off[i];
  for (int k = 0; k < 4; k++)
    if (m & (1 << k)) keys[w++] = ((unsigned long long)(unsigned)nb[k] << 32) | (unsigned)ea;
  for (int k = 0; k < 4; k++)
    if (m & (16 << k)) keys[w++] = ((unsigned long long)(unsigned)na[k] << 32) | (unsigned)eb;
}

__device__ double clamp01(double n) { return n <= 0 ? 0 : n >= 1 ? 1 : n; }

// dtn, dist_node2tri.h:14-129 (including its clamp of -e/c in region 6)
__device__ double dtn(const double f[9], const double p[3]) {
  double E0[3], E1[3], v0[3];
  for (int k = 0; k < 3; k++) {
    E0[k] = f[3 + k] - f[k];
    E1[k] = f[6 + k] - f[k];
    v0[k] = f[k] - p[k];
  }
  const double a = E0[0] * E0[0] + E0[1] * E0[1] + E0[2] * E0[2];
  const double b = E0[0] * E1[0] + E0[1] * E1[1] + E0[2] * E1[2];
  const double c = E1[0] * E1[0] + E1[1] * E1[1] + E1[2] * E1[2];
  const double d = E0[0] * v0[0] + E0[1] * v0[1] + E0[2] * v0[2];
  const double e = E1[0] * v0[0] + E1[1] * v0[1] + E1[2] * v0[2];
  const double det = a * c - b * b;
  double s = b * e - c * d, t = b * d - a * e;
  if (s + t < det) {
    if (s < 0) {
      if (t < 0 && d < 0) { s = clamp01(-d / a); t = 0; }
      else { s = 0; t = clamp01(-e / c); }
    } else if (t < 0) {
      s = clamp01(-d / a);
      t = 0;
    } else {
      const double inv = 1.0 / det;
      s *= inv;
      t *= inv;
    }
  } else {
    if (s < 0) {
      const double t0 = b + d, t1 = c + e;
      if (t1 > t0) { s = clamp01((t1 - t0) / (a - 2 * b + c)); t = 1 - s; }
      else { t = clamp01(-e / c); s = 0; }
    } else if (t < 0) {
      if (a + d > b + e) { s = clamp01((c + e - b - d) / (a - 2 * b + c)); t = 1 - s; }
      else { s = clamp01(-e / c); t = 0; }
    } else {
      s = clamp01((c + e - b - d) / (a - 2 * b + c));
      t = 1 - s;
    }
  }
  double r = 0;
  for (int k = 0; k < 3; k++) {
    const double dk = f[k] + s * E0[k] + t * E1[k] - p[k];
    r += dk * dk;
  }
  return r;
}

__global__ void k_closest(int n, const unsigned long long *__restrict__ keys,
                          const int *__restrict__ adj_off, const int *__restrict__ adj,
                          const int *__restrict__ faces, const double4 *__restrict__ xc,
                          int4 *__restrict__ imp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned long long key = keys[i];
  const int node = (int)(key >> 32), el = (int)(key & 0xffffffffULL);
  const double4 pp = xc[node];
  const double p[3] = {pp.x, pp.y, pp.z};
  int best = -1;
  double bestd = 0;
  for (int q = adj_off[el]; q < adj_off[el + 1]; q++) {
    const int fc = adj[q];
    double fx[9];
    for (int v = 0; v < 3; v++) {
      const double4 c = xc[faces[3 * fc + v]];
      fx[3 * v] = c.x; fx[3 * v + 1] = c.y; fx[3 * v + 2] = c.z;
    }
    const double dd = dtn(fx, p);
    if (q == adj_off[el] || dd < bestd) {
      best = fc;
      bestd = dd;
    }
  }
  if (best < 0) {
    imp[i] = make_int4(node, -1, -1, -1);
    return;
  }
  imp[i] = make_int4(node, faces[3 * best], faces[3 * best + 1], faces[3 * best + 2]);
}

// ---- point-triangle distance with first and second derivatives ----------------------
// x = (p, v0, v1, v2).  Vertex-vertex: |x_a - x_b|^2.
__device__ double pt_vv(const double x[12], int ia, int ib, double fd[12], double sd[144]) {
  double dsq = 0;
  for (int k = 0; k < 3; k++) {
    const double d = x[3 * ia + k] - x[3 * ib + k];
    fd[3 * ia + k] = 2 * d;
    fd[3 * ib + k] = -(2 * d);
    sd[(3 * ia + k) * 12 + 3 * ia + k] = 2;
    sd[(3 * ib + k) * 12 + 3 * ib + k] = 2;
    sd[(3 * ia + k) * 12 + 3 * ib + k] = -2;
    sd[(3 * ib + k) * 12 + 3 * ia + k] = -2;
    dsq += d * d;
  }
  return dsq;
}

// Point y[0..2] to the line (y[3..5], y[6..8]): dist^2 = f1 - g / f2 with
// f1 = |q1-p|^2, g = ((q1-p).(q2-q1))^2, f2 = |q2-q1|^2
// (vertex_edge_distance_and_derivs, point_triange_v2.h:152-232).
__device__ double pt_line(const double y[9], double fd[9], double sd[81]) {
  const double *P = y, *Q1 = y + 3, *Q2 = y + 6;
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
  double sp = 0, spd[9];
  for (int k = 0; k < 3; k++) {
    spd[k] = Q1[k] - Q2[k];
    spd[3 + k] = P[k] - 2 * Q1[k] + Q2[k];
    spd[6 + k] = Q1[k] - P[k];
    sp += (Q1[k] - P[k]) * (Q2[k] - Q1[k]);
  }
  // second derivatives of sp: -2 on (q1,q1), -1 on (p,q2), +1 on (p,q1), (q2,q1)
  auto spdd = [](int i, int j) -> double {
    if (i % 3 != j % 3) return 0.0;
    const int bi = i / 3, bj = j / 3;
    if (bi == 1 && bj == 1) return -2.0;
    if ((bi == 0 && bj == 2) || (bi == 2 && bj == 0)) return -1.0;
    if ((bi == 0 && bj == 1) || (bi == 1 && bj == 0) || (bi == 2 && bj == 1) || (bi == 1 && bj == 2))
      return 1.0;
    return 0.0;
  };
  const double g = sp * sp;
  double gd[9], f1d[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, f2d[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  double f2 = 0;
  for (int i = 0; i < 9; i++) gd[i] = 2 * sp * spd[i];
  for (int k = 0; k < 3; k++) {
    const double a = Q1[k] - P[k], b = Q2[k] - Q1[k];
    f2 += b * b;
    f1d[3 + k] = 2 * a;
    f1d[k] = -(2 * a);
    f2d[6 + k] = 2 * b;
    f2d[3 + k] = -(2 * b);
  }
  auto f1dd = [](int i, int j) -> double {
    if (i % 3 != j % 3) return 0.0;
    const int bi = i / 3, bj = j / 3;
    if (bi == 2 || bj == 2) return 0.0;
    return bi == bj ? 2.0 : -2.0;
  };
  auto f2dd = [](int i, int j) -> double {
    if (i % 3 != j % 3) return 0.0;
    const int bi = i / 3, bj = j / 3;
    if (bi == 0 || bj == 0) return 0.0;
    return bi == bj ? 2.0 : -2.0;
  };
  const double f2sq = f2 * f2, f2cu = f2sq * f2;
  for (int i = 0; i < 9; i++) {
    fd[i] = f1d[i] + (g * f2d[i] - f2 * gd[i]) / f2sq;
    for (int j = 0; j < 9; j++) {
      const double gdd = 2 * (spd[i] * spd[j] + sp * spdd(i, j));
      const double t1 = -2 * g * f2d[i] * f2d[j] / f2cu;
      const double t2 = (gd[i] * f2d[j] + gd[j] * f2d[i]) / f2sq;
      const double t3 = f1dd(i, j);
      const double t4 = g * f2dd(i, j) / f2sq;
      const double t5 = -gdd / f2;
      sd[i * 9 + j] = t1 + t2 + t3 + t4 + t5;
    }
  }
  return dist2;
}

// Point to the edge (ia, ib) of x[12]; the nearer endpoint is the origin.
__device__ double pt_ve(const double x[12], int ia, int ib, double fd[12], double sd[144]) {
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
  double y[9], yd[9], ydd[81];
  const int blk[3] = {0, ia, ib};
  for (int b = 0; b < 3; b++)
    for (int k = 0; k < 3; k++) y[3 * b + k] = x[3 * blk[b] + k];
  const double r = pt_line(y, yd, ydd);
  for (int bi = 0; bi < 3; bi++)
    for (int k = 0; k < 3; k++) {
      fd[3 * blk[bi] + k] = yd[3 * bi + k];
      for (int bj = 0; bj < 3; bj++)
        for (int l = 0; l < 3; l++)
          sd[(3 * blk[bi] + k) * 12 + 3 * blk[bj] + l] = ydd[(3 * bi + k) * 9 + 3 * bj + l];
    }
  return r;
}

// Interior region: |q|^2 with q = s v1 + t v2 + (1-s-t) v0 - p and the
// barycentric foot point s(x), t(x) of the plane (point_plane_distance,
// point_triange_v2.h:449-582).  The gradients of a..e come from their
// bilinear structure (a = e0.e0, b = e0.e1, c = e1.e1, d = e0.w, e = e1.w;
// e0 = v1-v0, e1 = v2-v0, w = v0-p); their Hessians are multiples of the
// identity per 3x3 block.
struct sel {
  int bp, bn;  // +x[block bp] - x[block bn]
};
__device__ void bil(sel A, sel C, const double ax[3], const double cx[3], double g[12],
                    double H[4][4]) {
  for (int i = 0; i < 12; i++) g[i] = 0;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) H[i][j] = 0;
  for (int k = 0; k < 3; k++) {
    g[3 * A.bp + k] += cx[k];
    g[3 * A.bn + k] -= cx[k];
    g[3 * C.bp + k] += ax[k];
    g[3 * C.bn + k] -= ax[k];
  }
  const int ab[2] = {A.bp, A.bn}, cb[2] = {C.bp, C.bn};
  const double sg[2] = {1.0, -1.0};
  for (int i = 0; i < 2; i++)
    for (int j = 0; j < 2; j++) {
      H[ab[i]][cb[j]] += sg[i] * sg[j];
      H[cb[j]][ab[i]] += sg[i] * sg[j];
    }
}

__device__ double pt_plane(const double x[12], double fd[12], double sd[144]) {
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
  const double det = a * c - b * b, det2 = det * det, det3 = det2 * det;
  const double inv = 1. / det;
  const double s = (b * e - c * d) * inv, t = (b * d - a * e) * inv;
  const double u = 1 - (s + t);
  double q[3], dist2 = 0;
  for (int k = 0; k < 3; k++) {
    q[k] = -P[k] + V1[k] * s + V2[k] * t + V0[k] * u;
    dist2 += q[k] * q[k];
  }
  const sel E0 = {2, 1}, E1 = {3, 1}, W = {1, 0};
  double ag[12], bg[12], cg[12], dg[12], eg[12];
  double aH[4][4], bH[4][4], cH[4][4], dH[4][4], eH[4][4];
  bil(E0, E0, e0, e0, ag, aH);
  bil(E0, E1, e0, e1, bg, bH);
  bil(E1, E1, e1, e1, cg, cH);
  bil(E0, W, e0, w, dg, dH);
  bil(E1, W, e1, w, eg, eH);
  double s1[12], t1[12], u1[12], det1[12], J[3][12];
  for (int i = 0; i < 12; i++) {
    det1[i] = c * ag[i] + a * cg[i] - 2 * b * bg[i];
    s1[i] = ((c * d - b * e) * det1[i]) / det2 + ((e * bg[i] + b * eg[i]) - (d * cg[i] + c * dg[i])) / det;
    t1[i] = ((a * e - b * d) * det1[i]) / det2 + ((d * bg[i] + b * dg[i]) - (a * eg[i] + e * ag[i])) / det;
    u1[i] = -(s1[i] + t1[i]);
  }
  for (int k = 0; k < 3; k++)
    for (int i = 0; i < 12; i++) {
      double v = V1[k] * s1[i] + V2[k] * t1[i] + V0[k] * u1[i];
      if (i == k) v -= 1;
      if (i == 3 + k) v += u;
      if (i == 6 + k) v += s;
      if (i == 9 + k) v += t;
      J[k][i] = v;
    }
  for (int i = 0; i < 12; i++) fd[i] = 2 * (q[0] * J[0][i] + q[1] * J[1][i] + q[2] * J[2][i]);
  const double sN = -(c * d) + b * e, tN = b * d - a * e;
  for (int i = 0; i < 12; i++)
    for (int j = 0; j < 12; j++) {
      const bool same = (i % 3) == (j % 3);
      const int bi = i / 3, bj = j / 3;
      const double a2 = same ? aH[bi][bj] : 0, b2 = same ? bH[bi][bj] : 0;
      const double c2 = same ? cH[bi][bj] : 0, d2 = same ? dH[bi][bj] : 0;
      const double e2 = same ? eH[bi][bj] : 0;
      const double dt2 = -2 * bg[i] * bg[j] + ag[j] * cg[i] + ag[i] * cg[j] + c * a2 - 2 * b * b2 + a * c2;
      const double s2 =
          (-(cg[j] * dg[i]) - cg[i] * dg[j] + bg[j] * eg[i] + bg[i] * eg[j] + e * b2 - d * c2 - c * d2 + b * e2) / det -
          ((det1[j] * (e * bg[i] - d * cg[i] - c * dg[i] + b * eg[i])) +
           (det1[i] * (e * bg[j] - d * cg[j] - c * dg[j] + b * eg[j])) + (sN * dt2)) / det2 +
          (2 * sN * det1[i] * det1[j]) / det3;
      const double t2 =
          (bg[j] * dg[i] + bg[i] * dg[j] - ag[j] * eg[i] - ag[i] * eg[j] - e * a2 + d * b2 + b * d2 - a * e2) / det -
          ((det1[j] * (-(e * ag[i]) + d * bg[i] + b * dg[i] - a * eg[i])) +
           (det1[i] * (-(e * ag[j]) + d * bg[j] + b * dg[j] - a * eg[j])) + (tN * dt2)) / det2 +
          (2 * tN * det1[i] * det1[j]) / det3;
      const double u2 = -(s2 + t2);
      double acc = 0;
      for (int k = 0; k < 3; k++) {
        double q2 = V1[k] * s2 + V2[k] * t2 + V0[k] * u2;
        if (i == 3 + k) q2 += u1[j];
        if (j == 3 + k) q2 += u1[i];
        if (i == 6 + k) q2 += s1[j];
        if (j == 6 + k) q2 += s1[i];
        if (i == 9 + k) q2 += t1[j];
        if (j == 9 + k) q2 += t1[i];
        acc += J[k][i] * J[k][j] + q[k] * q2;
      }
      sd[i * 12 + j] = 2 * acc;
    }
  return dist2;
}

// pt (point_triange_v2.h:589-841): Voronoi region of the closest feature.
__device__ double pt(const double x[12], double fd[12], double sd[144], double &s_out,
                     double &t_out) {
  for (int i = 0; i < 12; i++) fd[i] = 0;
  for (int i = 0; i < 144; i++) sd[i] = 0;
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
  double s = b * e - c * d, t = b * d - a * e, r;
  if (s + t <= det) {
    if (s < 0) {
      if (t < 0 && d < 0) {
        t = 0;
        if (-d >= a) { s = 1; r = pt_vv(x, 0, 2, fd, sd); }
        else { s = -d / a; r = pt_ve(x, 2, 1, fd, sd); }
      } else {
        s = 0;
        if (e >= 0) { t = 0; r = pt_vv(x, 0, 1, fd, sd); }
        else if (-e >= c) { t = 1; r = pt_vv(x, 0, 3, fd, sd); }
        else { t = -e / c; r = pt_ve(x, 3, 1, fd, sd); }
      }
    } else if (t < 0) {
      t = 0;
      if (d >= 0) { s = 0; r = pt_vv(x, 0, 1, fd, sd); }
      else if (-d >= a) { s = 1; r = pt_vv(x, 0, 2, fd, sd); }
      else { s = -d / a; r = pt_ve(x, 1, 2, fd, sd); }
    } else {
      const double inv = (1) / det;
      s *= inv;
      t *= inv;
      r = pt_plane(x, fd, sd);
    }
  } else {
    if (s < 0) {
      const double t0 = b + d, t1 = c + e;
      if (t1 > t0) {
        const double num = t1 - t0, den = a - 2 * b + c;
        if (num >= den) { s = 1; t = 0; r = pt_vv(x, 0, 2, fd, sd); }
        else { s = num / den; t = 1 - s; r = pt_ve(x, 2, 3, fd, sd); }
      } else {
        s = 0;
        if (t1 <= 0) { t = 1; r = pt_vv(x, 0, 3, fd, sd); }
        else if (e >= 0) { t = 0; r = pt_vv(x, 0, 1, fd, sd); }
        else { t = -e / c; r = pt_ve(x, 1, 3, fd, sd); }
      }
    } else if (t < 0) {
      const double t0 = b + e, t1 = a + d;
      if (t1 > t0) {
        const double num = t1 - t0, den = a - 2 * b + c;
        if (num >= den) { t = 1; s = 0; r = pt_vv(x, 0, 3, fd, sd); }
        else { t = num / den; s = 1 - t; r = pt_ve(x, 2, 3, fd, sd); }
      } else {
        t = 0;
        if (t1 <= 0) { s = 1; r = pt_vv(x, 0, 2, fd, sd); }
        else if (d >= 0) { s = 0; r = pt_vv(x, 0, 1, fd, sd); }
        else { s = -d / a; r = pt_ve(x, 1, 2, fd, sd); }
      }
    } else {
      const double num = c + e - b - d;
      if (num <= 0) { s = 0; t = 1; r = pt_vv(x, 0, 3, fd, sd); }
      else {
        const double den = a - 2 * b + c;
        if (num >= den) { s = 1; t = 0; r = pt_vv(x, 0, 2, fd, sd); }
        else { s = num / den; t = 1 - s; r = pt_ve(x, 2, 3, fd, sd); }
      }
    }
  }
  s_out = s;
  t_out = t;
  return r;
}

// Penalty response of one impact: staging = 12x12 LHS then the 12 rhs.
__global__ void __launch_bounds__(64)
    k_imp_unit(int n, const int4 *__restrict__ imp, const int *__restrict__ alt,
               const double4 *__restrict__ xc, double k, double eps2,
               double *__restrict__ ks, int *__restrict__ counts) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n) return;
  double *K = ks + (size_t)u * ICF_IMP_STAGE;
  const int4 id = imp[u];
  const int nid[4] = {id.x, id.y, id.z, id.w};
  bool any_active = false;
  for (int i = 0; i < 4; i++) any_active |= (nid[i] >= 0 && alt[nid[i]] >= 0);
  double x[12];
  bool ok = any_active && id.y >= 0;
  if (ok)
    for (int i = 0; i < 4; i++) {
      const double4 p = xc[nid[i]];
      x[3 * i] = p.x; x[3 * i + 1] = p.y; x[3 * i + 2] = p.z;
    }
  double fd[12], sd[144], s = 0, t = 0, dsq = 0;
  if (ok) dsq = pt(x, fd, sd, s, t);
  if (!ok || !(dsq > eps2)) {
    for (int i = 0; i < ICF_IMP_STAGE; i++) K[i] = 0;
    return;
  }
  const double w[3] = {1 - (s + t), s, t};
  const double F[3] = {k * 0.5 * fd[0], k * 0.5 * fd[1], k * 0.5 * fd[2]};
  for (int i = 0; i < 12; i++)
    for (int j = i; j < 12; j++) K[i * 12 + j] = K[j * 12 + i] = k * sd[i * 12 + j] / 2;
  for (int c = 0; c < 3; c++) {
    K[144 + c] = -F[c];
    for (int v = 0; v < 3; v++) K[144 + 3 + 3 * v + c] = w[v] * F[c];
  }
  atomicAdd(counts + 3, 1);
}

}  // namespace

int icf_launch_imp_unit(icf_ctx *ctx) {
  k_imp_unit<<<icf_blocks(ctx->n_imp, 64), 64, 0, ctx->stream>>>(
      ctx->n_imp, ctx->d_imp, ctx->d_alt, ctx->d_xc, ctx->prm.penaltyK,
      ctx->prm.DistanceEpsilon * ctx->prm.DistanceEpsilon, ctx->d_ks, ctx->d_counts);
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}

// Narrow phase + set expansion + closest face.  Leaves ctx->d_imp /
// ctx->n_imp set; the pattern must be rebuilt afterwards.
int icf_run_narrow_phase(icf_ctx *ctx, int n_pairs, int *n_impacts) {
  cudaStream_t s = ctx->stream;
  if (n_pairs == 0) {
    ctx->n_imp = 0;
    *n_impacts = 0;
    return ICF_OK;
  }
  // counts and offsets of the set bits
  int *d_cnt = nullptr, *d_off = nullptr;
  ICF_CUDA(ctx, cudaMallocAsync(&d_cnt, sizeof(int) * (n_pairs + 1), s));
  ICF_CUDA(ctx, cudaMallocAsync(&d_off, sizeof(int) * (n_pairs + 1), s));
  k_narrow<<<icf_blocks(n_pairs, 128), 128, 0, s>>>(n_pairs, ctx->d_pairs, ctx->d_selem, ctx->d_xc,
                                                   ctx->d_masks, d_cnt);
  ICF_CUDA(ctx, cudaGetLastError());
  ICF_CUDA(ctx, cudaMemsetAsync(d_cnt + n_pairs, 0, sizeof(int), s));
  size_t tb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb, d_cnt, d_off, n_pairs + 1, s);
  if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
  ICF_CUDA(ctx, cub::DeviceScan::ExclusiveSum(ctx->d_tmp, tb, d_cnt, d_off, n_pairs + 1, s));
  int total = 0;
  ICF_CUDA(ctx, cudaMemcpyAsync(&total, d_off + n_pairs, sizeof(int), cudaMemcpyDeviceToHost, s));
  ICF_CUDA(ctx, cudaStreamSynchronize(s));
  int nu = 0;
  if (total > 0) {
    unsigned long long *k0 = nullptr, *k1 = nullptr;
    int *d_nu = nullptr;
    ICF_CUDA(ctx, cudaMallocAsync(&k0, sizeof(unsigned long long) * total, s));
    ICF_CUDA(ctx, cudaMallocAsync(&k1, sizeof(unsigned long long) * total, s));
    ICF_CUDA(ctx, cudaMallocAsync(&d_nu, sizeof(int), s));
    k_expand<<<icf_blocks(n_pairs, 128), 128, 0, s>>>(n_pairs, ctx->d_pairs, ctx->d_selem,
                                                     ctx->d_masks, d_off, k0);
    tb = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, tb, k0, k1, total, 0, 64, s);
    if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
    ICF_CUDA(ctx, cub::DeviceRadixSort::SortKeys(ctx->d_tmp, tb, k0, k1, total, 0, 64, s));
    tb = 0;
    cub::DeviceSelect::Unique(nullptr, tb, k1, k0, d_nu, total, s);
    if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
    ICF_CUDA(ctx, cub::DeviceSelect::Unique(ctx->d_tmp, tb, k1, k0, d_nu, total, s));
    ICF_CUDA(ctx, cudaMemcpyAsync(&nu, d_nu, sizeof(int), cudaMemcpyDeviceToHost, s));
    ICF_CUDA(ctx, cudaStreamSynchronize(s));
    if (nu > ctx->imp_cap) {
      if (ctx->d_imp) cudaFree(ctx->d_imp);
      ctx->d_imp = nullptr;
      ICF_CUDA(ctx, cudaMalloc(&ctx->d_imp, sizeof(int4) * (size_t)(2 * nu)));
      ctx->imp_cap = 2 * nu;
    }
    k_closest<<<icf_blocks(nu, 128), 128, 0, s>>>(nu, k0, ctx->d_adj_off, ctx->d_adj, ctx->d_faces,
                                                 ctx->d_xc, ctx->d_imp);
    ICF_CUDA(ctx, cudaGetLastError());
    ICF_CUDA(ctx, cudaFreeAsync(k0, s));
    ICF_CUDA(ctx, cudaFreeAsync(k1, s));
    ICF_CUDA(ctx, cudaFreeAsync(d_nu, s));
  }
  ICF_CUDA(ctx, cudaFreeAsync(d_cnt, s));
  ICF_CUDA(ctx, cudaFreeAsync(d_off, s));
  ICF_CUDA(ctx, cudaStreamSynchronize(s));
  ctx->n_imp = nu;
  *n_impacts = nu;
  return ICF_OK;
}
