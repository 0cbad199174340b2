// icf_contact_deriv.cu -- penalty response of the impacts, one warp per impact.
//
// kCollisionResponseForce (collision_response.h:38-127) needs the gradient
// and Hessian of the squared point-triangle distance d2(x), x = (p, v0, v1,
// v2), in the Voronoi region found by k_imp_classify (icf_contact.cu):
//   vertex region  d2 = |p - v|^2
//   edge region    d2 = f1 - g / f2,  f1 = |q1-p|^2, g = ((q1-p).(q2-q1))^2,
//                  f2 = |q2-q1|^2   (point_triange_v2.h:152-232)
//   interior       the squared distance to the triangle's plane
//                  (point_plane_distance, :449-582)
// In the interior the reference differentiates d2 = |q|^2 through the
// barycentrics s(x), t(x) of the foot point.  The same function is
// d2 = D^2 / S with D = a . N, S = N . N, N = e0 x e1, a = p - v0,
// e0 = v1 - v0, e1 = v2 - v0, whose Hessian has the closed form
//   H = 2 gD gD^T / S + 2 D HD / S - 2 D (gD gS^T + gS gD^T) / S^2
//       - D^2 HS / S^2 + 2 D^2 gS gS^T / S^3,
// gD, gS the gradients and HD, HS the Hessians of D and S: HD is a
// cross-product matrix per vertex-block pair (D is trilinear in a, e0, e1),
// HS follows from S = |e0|^2 |e1|^2 - (e0.e1)^2.  About 40 operations per
// entry instead of some 200; the two forms agree to rounding (1e-14 of the
// largest entry on random interior cases).
//
// The 32 lanes of a warp share the per-impact setup through shared memory.
// The Hessian K = k/2 d2'' goes straight to the records of the impact's
// contribution codes, at their positions in the slot-sorted list
// (icf_internal.cuh, ICF_IMP_REC): a lane per record entry (10 vertex pairs x
// 9 entries), each written once; a diagonal block's lower entries are
// evaluated at (column, row), so the block is symmetric bit for bit.  On the
// diagonal codes the record also carries the vertex's rhs from (-F, w0 F,
// w1 F, w2 F), F = k/2 d(d2)/dp, w = (1-s-t, s, t); the four vertex forces
// also go to a per-impact force record (for the node forces).
#include "icf_internal.cuh"

namespace {

constexpr int WARPS = 4;

// coefficients of vertex block b (p, v0, v1, v2) in a = p - v0,
// e0 = v1 - v0, e1 = v2 - v0
__device__ __forceinline__ double cA(int b) { return b == 0 ? 1.0 : (b == 1 ? -1.0 : 0.0); }
__device__ __forceinline__ double cE0(int b) { return b == 2 ? 1.0 : (b == 1 ? -1.0 : 0.0); }
__device__ __forceinline__ double cE1(int b) { return b == 3 ? 1.0 : (b == 1 ? -1.0 : 0.0); }

// Interior region, per impact: the gradients of D and S, the rank-two part's
// factors u = c1 gD + c3 gS, w = c3 gD + c5 gS (so that c1 gD gD^T + c3 (gD gS^T
// + gS gD^T) + c5 gS gS^T = u gD^T + w gS^T), the Hessian blocks of S over
// (e0, e0), (e1, e1), (e0, e1), and per vertex-block pair (bi, bj) the vector W
// with HD's block = [W]x.
struct PlaneSetup {
  double gD[12], gS[12], u[12], w[12];
  double h00[9], h11[9], h01[9];
  double W[16][3];
};

struct LineSetup {
  double sp, g, f2, f2sq, f2cu;
  double spd[9], gd[9], f1d[9], f2d[9];
};

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

// component k of a 3-vector held in registers (selects, no local memory)
__device__ __forceinline__ double pick3(const double v[3], int k) { return k == 0 ? v[0] : (k == 1 ? v[1] : v[2]); }

// Entry (ci, cj) of the cross-product matrix [w]x (w x y = [w]x y).
__device__ __forceinline__ double cross_entry(const double w[3], int ci, int cj) {
  if (ci == cj) return 0.0;
  const double wk = pick3(w, 3 - ci - cj);
  return ((cj - ci + 3) % 3 == 1) ? -wk : wk;
}

// Closed-form Hessian entry (I, J) of the squared distance to the plane:
// u_I gD_J + w_I gS_J + c2 HD_IJ + c4 HS_IJ.
__device__ __forceinline__ double plane_entry(const PlaneSetup &S, double c2, double c4, int I, int J) {
  const int bi = I / 3, bj = J / 3, ci = I % 3, cj = J % 3;
  const double pi0 = cE0(bi), pj0 = cE0(bj), pi1 = cE1(bi), pj1 = cE1(bj);
  const double hd = cross_entry(S.W[4 * bi + bj], ci, cj);
  const double hs = pi0 * pj0 * S.h00[3 * ci + cj] + pi1 * pj1 * S.h11[3 * ci + cj] +
                    pi0 * pj1 * S.h01[3 * ci + cj] + pi1 * pj0 * S.h01[3 * cj + ci];
  return S.u[I] * S.gD[J] + S.w[I] * S.gS[J] + c2 * hd + c4 * hs;
}

// record entry slot (0..89) -> vertex pair (bA <= bB) and entry (r, c) of
// its 3x3 block: the four diagonal pairs, then the six off-diagonal ones
__constant__ int kPairA[10] = {0, 1, 2, 3, 0, 0, 0, 1, 1, 2};
__constant__ int kPairB[10] = {0, 1, 2, 3, 1, 2, 3, 2, 3, 3};
__device__ __forceinline__ void slot_entry(int sl, int &bA, int &bB, int &r, int &c) {
  const int pi = sl / 9, e = sl % 9;
  bA = kPairA[pi];
  bB = kPairB[pi];
  r = e / 3;
  c = e % 3;
}

__global__ void __launch_bounds__(32 * WARPS)
    k_imp_deriv(int n, const int4 *__restrict__ imp, const double4 *__restrict__ xc,
                const int4 *__restrict__ ci, const double4 *__restrict__ cd, double kpen,
                const int *__restrict__ pos, double *__restrict__ rec, double *__restrict__ frc) {
  __shared__ PlaneSetup sP[WARPS];
  __shared__ LineSetup sL[WARPS];
  __shared__ double sx[WARPS][12];
  __shared__ double sfd[WARPS][3];
  __shared__ int sPos[WARPS][16];
  const int wl = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int u = blockIdx.x * WARPS + wl;
  if (u >= n) return;  // uniform per warp
  const int *P = pos + 16 * (size_t)u;
  const int4 c = ci[u];
  if (lane < 16) sPos[wl][lane] = P[lane];
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
  const int kind = c.x;
  double c2 = 0, c4 = 0;  // interior: the scalars of HD and HS
  if (kind == 1) {  // vertex: d2 = |p - x_b|^2
    if (lane < 3) sfd[wl][lane] = 2 * (x[lane] - x[3 * c.z + lane]);
  } else if (kind == 2) {  // edge (ia nearer, ib)
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
  } else {  // interior: d2 = D^2 / S
    PlaneSetup &S = sP[wl];
    double a[3], e0[3], e1[3], N[3], e1xa[3], axe0[3], e1xN[3], Nxe0[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      a[k] = x[k] - x[3 + k];
      e0[k] = x[6 + k] - x[3 + k];
      e1[k] = x[9 + k] - x[3 + k];
    }
#define CROSS(o, u_, v_)                          \
  o[0] = u_[1] * v_[2] - u_[2] * v_[1];           \
  o[1] = u_[2] * v_[0] - u_[0] * v_[2];           \
  o[2] = u_[0] * v_[1] - u_[1] * v_[0];
    CROSS(N, e0, e1)
    CROSS(e1xa, e1, a)
    CROSS(axe0, a, e0)
    CROSS(e1xN, e1, N)
    CROSS(Nxe0, N, e0)
#undef CROSS
    const double D = a[0] * N[0] + a[1] * N[1] + a[2] * N[2];
    const double Sv = N[0] * N[0] + N[1] * N[1] + N[2] * N[2];
    const double iS = 1.0 / Sv;
    const double c1 = 2.0 * iS, c3 = -2.0 * D * iS * iS, c5 = 2.0 * D * D * iS * iS * iS;
    c2 = 2.0 * D * iS;
    c4 = -D * D * iS * iS;
    if (lane < 12) {
      const int b = lane / 3, k = lane % 3;
      const double gd = cA(b) * pick3(N, k) + cE0(b) * pick3(e1xa, k) + cE1(b) * pick3(axe0, k);
      const double gs = 2.0 * (cE0(b) * pick3(e1xN, k) + cE1(b) * pick3(Nxe0, k));
      S.gD[lane] = gd;
      S.gS[lane] = gs;
      S.u[lane] = c1 * gd + c3 * gs;
      S.w[lane] = c3 * gd + c5 * gs;
    } else if (lane < 21) {  // HS blocks, S = |e0|^2 |e1|^2 - (e0.e1)^2
      const int r = (lane - 12) / 3, q = (lane - 12) % 3;
      const double dl = r == q ? 1.0 : 0.0;
      const double e00 = e0[0] * e0[0] + e0[1] * e0[1] + e0[2] * e0[2];
      const double e11 = e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2];
      const double e01 = e0[0] * e1[0] + e0[1] * e1[1] + e0[2] * e1[2];
      const double e0r = pick3(e0, r), e0q = pick3(e0, q), e1r = pick3(e1, r), e1q = pick3(e1, q);
      S.h00[3 * r + q] = 2.0 * (e11 * dl - e1r * e1q);
      S.h11[3 * r + q] = 2.0 * (e00 * dl - e0r * e0q);
      S.h01[3 * r + q] = 4.0 * e0r * e1q - 2.0 * e1r * e0q - 2.0 * e01 * dl;
    }
    // W per vertex-block pair: D is trilinear in (a, e0, e1), so HD's block
    // (bi, bj) is [W]x, W = -e1 (ai pj0 - pi0 aj) + e0 (ai pj1 - pi1 aj)
    // - a (pi0 pj1 - pi1 pj0)
    for (int l = lane; l < 48; l += 32) {
      const int pr = l / 3, k = l % 3, bi = pr / 4, bj = pr % 4;
      const double ai = cA(bi), aj = cA(bj), pi0 = cE0(bi), pj0 = cE0(bj), pi1 = cE1(bi), pj1 = cE1(bj);
      const double al = ai * pj0 - pi0 * aj, be = ai * pj1 - pi1 * aj, ga = pi0 * pj1 - pi1 * pj0;
      S.W[pr][k] = -pick3(e1, k) * al + pick3(e0, k) * be - pick3(a, k) * ga;
    }
    // d(d2)/dp = 2 D N / S
    if (lane < 3) sfd[wl][lane] = c2 * pick3(N, lane);
  }
  __syncwarp();
  // one lane per record entry: pair (bA, bB), entry (r, c); the three
  // entries of a lane are computed first and stored after, so that their
  // shared-memory reads overlap
  double val[3];
  long long dst[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const int sl = lane + 32 * k;
    val[k] = 0.0;
    dst[k] = -1;
    if (sl < 90) {
      int bA, bB, r, cc;
      slot_entry(sl, bA, bB, r, cc);
      int I = 3 * bA + r, J = 3 * bB + cc;
      if (I > J) {  // lower entry of a diagonal block: its mirror
        const int t = I;
        I = J;
        J = t;
      }
      double v = 0;
      if (kind == 1) {
        const int vb = c.z, bI = I / 3, bJ = J / 3;
        if (I % 3 == J % 3 && (bI == 0 || bI == vb) && (bJ == 0 || bJ == vb)) v = (bI == bJ) ? 2.0 : -2.0;
      } else if (kind == 2) {
        const int ia = c.y, ib = c.z, bI = I / 3, bJ = J / 3;
        const int pI = bI == 0 ? 0 : (bI == ia ? 1 : (bI == ib ? 2 : -1));
        const int pJ = bJ == 0 ? 0 : (bJ == ia ? 1 : (bJ == ib ? 2 : -1));
        if (pI >= 0 && pJ >= 0) v = line_entry(sL[wl], 3 * pI + I % 3, 3 * pJ + J % 3);
      } else {
        v = plane_entry(sP[wl], c2, c4, I, J);
      }
      val[k] = kpen * v / 2;
      // the code of the pair, taken either way round (none: an anchored vertex)
      const int q = sPos[wl][4 * bA + bB];
      if (q >= 0) {
        dst[k] = ICF_IMP_REC * (long long)q + 3 * r + cc;
      } else if (bA != bB) {
        const int q2 = sPos[wl][4 * bB + bA];
        if (q2 >= 0) dst[k] = ICF_IMP_REC * (long long)q2 + 3 * cc + r;
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 3; k++)
    if (dst[k] >= 0) rec[dst[k]] = val[k];
  // vertex forces (-F, w0 F, w1 F, w2 F), F = k/2 d(d2)/dp, w = (1-s-t, s, t)
  // (collision_response.h:89-109): into the force record, and as the rhs of
  // the vertex's diagonal code
  if (lane < 12) {
    const double s = cl.x, t = cl.y;
    const int comp = lane % 3, blk = lane / 3;
    const double F = hk * sfd[wl][comp];
    const double f = blk == 0 ? -F : (blk == 1 ? (1 - (s + t)) : (blk == 2 ? s : t)) * F;
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
