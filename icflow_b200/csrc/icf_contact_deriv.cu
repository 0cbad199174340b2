// icf_contact_deriv.cu -- penalty response of the impacts, one warp per impact.
//
// kCollisionResponseForce (collision_response.h:38-127) needs the gradient
// and Hessian of the squared point-triangle distance d2(x), x = (p, v0, v1,
// v2), in the Voronoi region found by k_imp_classify (icf_contact.cu):
//   vertex region  d2 = |p - v|^2
//   edge region    d2 = f1 - g / f2,  f1 = |q1-p|^2, g = ((q1-p).(q2-q1))^2,
//                  f2 = |q2-q1|^2   (point_triange_v2.h:152-232)
//   interior       d2 = |q|^2, q = s v1 + t v2 + (1-s-t) v0 - p with the
//                  barycentrics s(x), t(x) of the foot point
//                  (point_plane_distance, :449-582)
// The 32 lanes of a warp share the per-impact setup through shared memory and
// each evaluates 2-3 of the 78 entries of the symmetric Hessian (:111-114).
// K = k/2 d2'' goes straight to the records of the impact's contribution
// codes, at their positions in the slot-sorted list (icf_internal.cuh,
// ICF_IMP_REC): the 3x3 block of each code's vertex pair, and, on the
// diagonal codes, the vertex's rhs from (-F, w0 F, w1 F, w2 F),
// F = k/2 d(d2)/dp, w = (1-s-t, s, t); the four vertex forces also go to a
// per-impact force record (for the node forces).
#include "icf_internal.cuh"

namespace {

constexpr int WARPS = 4;

// sign of block b in the selectors e0 = v1 - v0, e1 = v2 - v0, w = v0 - p
__device__ __forceinline__ double sgE0(int b) { return b == 2 ? 1.0 : (b == 1 ? -1.0 : 0.0); }
__device__ __forceinline__ double sgE1(int b) { return b == 3 ? 1.0 : (b == 1 ? -1.0 : 0.0); }
__device__ __forceinline__ double sgW(int b) { return b == 1 ? 1.0 : (b == 0 ? -1.0 : 0.0); }

struct PlaneSetup {
  double a, b, c, d, e, det, s, t, u, idet, idet2, idet3, sN, tN;
  double V[3][3];  // v0, v1, v2
  double q[3];
  double ag[12], bg[12], cg[12], dg[12], eg[12], det1[12], s1[12], t1[12], u1[12];
  double J[3][12];
};

struct LineSetup {
  double sp, g, f2, f2sq, f2cu;
  double spd[9], gd[9], f1d[9], f2d[9];
};

__device__ double plane_entry(const PlaneSetup &S, int i, int j) {
  const bool same = (i % 3) == (j % 3);
  const int bi = i / 3, bj = j / 3;
  double a2 = 0, b2 = 0, c2 = 0, d2 = 0, e2 = 0;
  if (same) {
    a2 = 2.0 * sgE0(bi) * sgE0(bj);
    b2 = sgE0(bi) * sgE1(bj) + sgE1(bi) * sgE0(bj);
    c2 = 2.0 * sgE1(bi) * sgE1(bj);
    d2 = sgE0(bi) * sgW(bj) + sgW(bi) * sgE0(bj);
    e2 = sgE1(bi) * sgW(bj) + sgW(bi) * sgE1(bj);
  }
  const double a = S.a, b = S.b, c = S.c, d = S.d, e = S.e;
  const double dt2 = -2 * S.bg[i] * S.bg[j] + S.ag[j] * S.cg[i] + S.ag[i] * S.cg[j] + c * a2 - 2 * b * b2 + a * c2;
  const double s2 =
      (-(S.cg[j] * S.dg[i]) - S.cg[i] * S.dg[j] + S.bg[j] * S.eg[i] + S.bg[i] * S.eg[j] + e * b2 - d * c2 -
       c * d2 + b * e2) * S.idet -
      ((S.det1[j] * (e * S.bg[i] - d * S.cg[i] - c * S.dg[i] + b * S.eg[i])) +
       (S.det1[i] * (e * S.bg[j] - d * S.cg[j] - c * S.dg[j] + b * S.eg[j])) + (S.sN * dt2)) * S.idet2 +
      (2 * S.sN * S.det1[i] * S.det1[j]) * S.idet3;
  const double t2 =
      (S.bg[j] * S.dg[i] + S.bg[i] * S.dg[j] - S.ag[j] * S.eg[i] - S.ag[i] * S.eg[j] - e * a2 + d * b2 +
       b * d2 - a * e2) * S.idet -
      ((S.det1[j] * (-(e * S.ag[i]) + d * S.bg[i] + b * S.dg[i] - a * S.eg[i])) +
       (S.det1[i] * (-(e * S.ag[j]) + d * S.bg[j] + b * S.dg[j] - a * S.eg[j])) + (S.tN * dt2)) * S.idet2 +
      (2 * S.tN * S.det1[i] * S.det1[j]) * S.idet3;
  const double u2 = -(s2 + t2);
  double acc = 0;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    double q2 = S.V[1][k] * s2 + S.V[2][k] * t2 + S.V[0][k] * u2;
    if (i == 3 + k) q2 += S.u1[j];
    if (j == 3 + k) q2 += S.u1[i];
    if (i == 6 + k) q2 += S.s1[j];
    if (j == 6 + k) q2 += S.s1[i];
    if (i == 9 + k) q2 += S.t1[j];
    if (j == 9 + k) q2 += S.t1[i];
    acc += S.J[k][i] * S.J[k][j] + S.q[k] * q2;
  }
  return 2 * acc;
}

// Hessian entry (i, j) of f1 - g / f2 over y = (p, q1, q2)
__device__ double line_entry(const LineSetup &L, int i, int j) {
  const bool same = (i % 3) == (j % 3);
  const int bi = i / 3, bj = j / 3;
  double spdd = 0, f1dd = 0, f2dd = 0;
  if (same) {
    if (bi == 1 && bj == 1) spdd = -2.0;
    else if ((bi == 0 && bj == 2) || (bi == 2 && bj == 0)) spdd = -1.0;
    else if (bi != bj) spdd = 1.0;
    if (bi != 2 && bj != 2) f1dd = (bi == bj) ? 2.0 : -2.0;
    if (bi != 0 && bj != 0) f2dd = (bi == bj) ? 2.0 : -2.0;
  }
  const double gdd = 2 * (L.spd[i] * L.spd[j] + L.sp * spdd);
  const double t1 = -2 * L.g * L.f2d[i] * L.f2d[j] / L.f2cu;
  const double t2 = (L.gd[i] * L.f2d[j] + L.gd[j] * L.f2d[i]) / L.f2sq;
  const double t4 = L.g * f2dd / L.f2sq;
  const double t5 = -gdd / L.f2;
  return t1 + t2 + f1dd + t4 + t5;
}

// Upper-triangle entry e (0..77) of a 12x12 matrix: (I, J), I <= J.
__device__ __forceinline__ void upper_ij(int e, int &I, int &J) {
  int i = 0, start = 0;
  while (e >= start + 12 - i) {
    start += 12 - i;
    i++;
  }
  I = i;
  J = i + (e - start);
}

// Entry (I, J) of the staged Hessian goes to the record of the code of vertex
// pair (I/3, J/3) at (I%3, J%3); pairs without a code (an anchored vertex, or
// the pair taken the other way round) are skipped.
__device__ __forceinline__ void put(const int *P, double *rec, int I, int J, double v) {
  const int q = P[4 * (I / 3) + J / 3];
  if (q >= 0) rec[ICF_IMP_REC * (size_t)q + 3 * (I % 3) + (J % 3)] = v;
}

__global__ void __launch_bounds__(32 * WARPS)
    k_imp_deriv(int n, const int4 *__restrict__ imp, const double4 *__restrict__ xc,
                const int4 *__restrict__ ci, const double4 *__restrict__ cd, double kpen,
                const int *__restrict__ pos, double *__restrict__ rec, double *__restrict__ frc) {
  __shared__ PlaneSetup sP[WARPS];
  __shared__ LineSetup sL[WARPS];
  __shared__ double sx[WARPS][12];
  __shared__ double sfd[WARPS][3];
  const int wl = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int u = blockIdx.x * WARPS + wl;
  if (u >= n) return;  // uniform per warp
  const int *P = pos + 16 * (size_t)u;
  const int4 c = ci[u];
  if (c.x < 0) {  // no response: zero records, zero forces
    for (int e = lane; e < 16 * ICF_IMP_REC; e += 32) {
      const int q = P[e / ICF_IMP_REC];
      if (q >= 0) rec[ICF_IMP_REC * (size_t)q + e % ICF_IMP_REC] = 0.0;
    }
    if (lane < 12) frc[12 * (size_t)u + lane] = 0.0;
    return;
  }
  const double4 cl = cd[u];
  const int4 id = imp[u];
  if (lane < 4) {
    const int nd = lane == 0 ? id.x : lane == 1 ? id.y : lane == 2 ? id.z : id.w;
    const double4 p = xc[nd];
    sx[wl][3 * lane] = p.x;
    sx[wl][3 * lane + 1] = p.y;
    sx[wl][3 * lane + 2] = p.z;
  }
  __syncwarp();
  const double *x = sx[wl];
  const double hk = kpen * 0.5;

  if (c.x == 1) {  // vertex: d2 = |p - x_b|^2
    const int vb = c.z;
    if (lane < 3) sfd[wl][lane] = 2 * (x[lane] - x[3 * vb + lane]);
    for (int e = lane; e < 78; e += 32) {
      int I, J;
      upper_ij(e, I, J);
      const int bI = I / 3, bJ = J / 3;
      double v = 0;
      if (I % 3 == J % 3 && (bI == 0 || bI == vb) && (bJ == 0 || bJ == vb)) v = (bI == bJ) ? 2.0 : -2.0;
      v = kpen * v / 2;
      put(P, rec, I, J, v);
      if (I != J) put(P, rec, J, I, v);
    }
  } else if (c.x == 2) {  // edge (ia nearer, ib)
    const int ia = c.y, ib = c.z;
    LineSetup &L = sL[wl];
    if (lane == 0) {
      const double *Pp = x, *Q1 = x + 3 * ia, *Q2 = x + 3 * ib;
      double sp = 0, f2 = 0;
      for (int k = 0; k < 3; k++) {
        L.spd[k] = Q1[k] - Q2[k];
        L.spd[3 + k] = Pp[k] - 2 * Q1[k] + Q2[k];
        L.spd[6 + k] = Q1[k] - Pp[k];
        sp += (Q1[k] - Pp[k]) * (Q2[k] - Q1[k]);
        const double a = Q1[k] - Pp[k], b = Q2[k] - Q1[k];
        f2 += b * b;
        L.f1d[3 + k] = 2 * a;
        L.f1d[k] = -(2 * a);
        L.f1d[6 + k] = 0;
        L.f2d[6 + k] = 2 * b;
        L.f2d[3 + k] = -(2 * b);
        L.f2d[k] = 0;
      }
      L.sp = sp;
      L.g = sp * sp;
      L.f2 = f2;
      L.f2sq = f2 * f2;
      L.f2cu = L.f2sq * f2;
      for (int i = 0; i < 9; i++) L.gd[i] = 2 * sp * L.spd[i];
      for (int k = 0; k < 3; k++)
        sfd[wl][k] = L.f1d[k] + (L.g * L.f2d[k] - L.f2 * L.gd[k]) / L.f2sq;
    }
    __syncwarp();
    for (int e = lane; e < 78; e += 32) {
      int I, J;
      upper_ij(e, I, J);
      const int bI = I / 3, bJ = J / 3;
      const int pI = bI == 0 ? 0 : (bI == ia ? 1 : (bI == ib ? 2 : -1));
      const int pJ = bJ == 0 ? 0 : (bJ == ia ? 1 : (bJ == ib ? 2 : -1));
      double v = 0;
      if (pI >= 0 && pJ >= 0) v = line_entry(L, 3 * pI + I % 3, 3 * pJ + J % 3);
      v = kpen * v / 2;
      put(P, rec, I, J, v);
      if (I != J) put(P, rec, J, I, v);
    }
  } else {  // interior
    PlaneSetup &S = sP[wl];
    // the scalars of point_plane_distance, on every lane (no round trip)
    double e0[3], e1[3], w[3];
    for (int k = 0; k < 3; k++) {
      e0[k] = -x[3 + k] + x[6 + k];
      e1[k] = -x[3 + k] + x[9 + k];
      w[k] = -x[k] + x[3 + k];
    }
    const double a = e0[0] * e0[0] + e0[1] * e0[1] + e0[2] * e0[2];
    const double b = e1[1] * e0[1] + e1[2] * e0[2] + e0[0] * e1[0];
    const double c2 = e1[1] * e1[1] + e1[2] * e1[2] + e1[0] * e1[0];
    const double d = w[0] * e0[0] + w[1] * e0[1] + w[2] * e0[2];
    const double e = e1[1] * w[1] + e1[2] * w[2] + w[0] * e1[0];
    const double det = a * c2 - b * b;
    const double idet = 1.0 / det, idet2 = idet * idet, idet3 = idet2 * idet;
    const double ss = (b * e - c2 * d) * idet, tt = (b * d - a * e) * idet, uu = 1 - (ss + tt);
    if (lane == 0) {
      S.a = a; S.b = b; S.c = c2; S.d = d; S.e = e;
      S.det = det; S.idet = idet; S.idet2 = idet2; S.idet3 = idet3;
      S.s = ss; S.t = tt; S.u = uu;
      S.sN = -(c2 * d) + b * e;
      S.tN = b * d - a * e;
    }
    if (lane < 9) S.V[lane / 3][lane % 3] = x[3 + lane];
    if (lane < 3) S.q[lane] = -x[lane] + x[6 + lane] * ss + x[9 + lane] * tt + x[3 + lane] * uu;
    if (lane < 12) {
      const int i = lane, bi = i / 3, k = i % 3;
      const double ag = 2.0 * sgE0(bi) * e0[k];
      const double bg = sgE0(bi) * e1[k] + sgE1(bi) * e0[k];
      const double cg = 2.0 * sgE1(bi) * e1[k];
      const double dg = sgE0(bi) * w[k] + sgW(bi) * e0[k];
      const double eg = sgE1(bi) * w[k] + sgW(bi) * e1[k];
      S.ag[i] = ag; S.bg[i] = bg; S.cg[i] = cg; S.dg[i] = dg; S.eg[i] = eg;
      const double det1 = c2 * ag + a * cg - 2 * b * bg;
      const double s1 = ((c2 * d - b * e) * det1) * idet2 + ((e * bg + b * eg) - (d * cg + c2 * dg)) * idet;
      const double t1 = ((a * e - b * d) * det1) * idet2 + ((d * bg + b * dg) - (a * eg + e * ag)) * idet;
      S.det1[i] = det1;
      S.s1[i] = s1;
      S.t1[i] = t1;
      S.u1[i] = -(s1 + t1);
      for (int kk = 0; kk < 3; kk++) {
        double v = x[6 + kk] * s1 + x[9 + kk] * t1 + x[3 + kk] * (-(s1 + t1));
        if (i == kk) v -= 1;
        if (i == 3 + kk) v += uu;
        if (i == 6 + kk) v += ss;
        if (i == 9 + kk) v += tt;
        S.J[kk][i] = v;
      }
    }
    __syncwarp();
    if (lane < 3) sfd[wl][lane] = 2 * (S.q[0] * S.J[0][lane] + S.q[1] * S.J[1][lane] + S.q[2] * S.J[2][lane]);
    for (int en = lane; en < 78; en += 32) {
      int I, J;
      upper_ij(en, I, J);
      const double v = kpen * plane_entry(S, I, J) / 2;
      put(P, rec, I, J, v);
      if (I != J) put(P, rec, J, I, v);
    }
  }
  __syncwarp();
  // vertex forces (-F, w0 F, w1 F, w2 F), F = k/2 d(d2)/dp, w = (1-s-t, s, t)
  // (collision_response.h:89-109): into the force record, and as the rhs of
  // the vertex's diagonal code
  if (lane < 12) {
    const double s = cl.x, t = cl.y;
    const double wv[3] = {1 - (s + t), s, t};
    const int comp = lane % 3, blk = lane / 3;
    const double F = hk * sfd[wl][comp];
    const double f = blk == 0 ? -F : wv[blk - 1] * F;
    frc[12 * (size_t)u + lane] = f;
    const int q = P[5 * blk];
    if (q >= 0) rec[ICF_IMP_REC * (size_t)q + 9 + comp] = f;
  } else if (lane < 28) {  // off-diagonal codes carry no rhs
    const int pr = lane - 12;
    const int q = P[pr];
    if ((pr >> 2) != (pr & 3) && q >= 0)
      for (int k = 0; k < 3; k++) rec[ICF_IMP_REC * (size_t)q + 9 + k] = 0.0;
  }
}

}  // namespace

int icf_launch_imp_deriv(icf_ctx *ctx, const int4 *cls_i, const double4 *cls_d, cudaStream_t stream) {
  return icf_launch_imp_deriv_bufs(ctx, ctx->d_xc, cls_i, cls_d, ctx->d_ks, stream);
}

// Derivative kernel with caller-chosen buffers (the allocation-free entry
// point passes its own staging).
int icf_launch_imp_deriv_bufs(icf_ctx *ctx, const double4 *xc, const int4 *cls_i, const double4 *cls_d,
                              double *ks, cudaStream_t stream) {
  k_imp_deriv<<<icf_blocks(ctx->n_imp, WARPS), 32 * WARPS, 0, stream>>>(
      ctx->n_imp, ctx->d_imp, xc, cls_i, cls_d, ctx->prm.penaltyK, ctx->d_imp_pos, ks,
      icf_imp_forces(ks, ctx->n_imp));
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}
