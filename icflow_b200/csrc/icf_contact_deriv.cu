// icf_contact_deriv.cu -- penalty response of the impacts, two impacts per warp.
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
// Sixteen lanes share an impact's setup through shared memory.
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
  double W[30];  // [3 pair + k], pairs (bi <= bj) in slot order
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


// Record entry slots (0..89): vertex pair (bA <= bB; the four diagonal
// pairs, then the six off-diagonal ones) and entry (r, c) of its 3x3 block.
// Everything an entry needs that depends on the slot alone is tabulated at
// compile time (kSlots):
//   a: I | J << 4 (the evaluated entry, I <= J: a diagonal block's lower
//      entries are taken at their mirror) | HD's index in W (3 pair + k)
//      << 8 | (HD's sign + 1) << 14
//   b: 3 ci + cj | (3 cj + ci) << 4 | the coefficients + 1 of HS's four
//      terms (pi0 pj0, pi1 pj1, pi0 pj1, pi1 pj0) << 8, 10, 12, 14
//   c: the code index of (bA, bB) | of (bB, bA) << 4 | offset 3 r + c in the
//      first's record << 8 | 3 c + r in the second's << 12
//   d: r | c << 2 | bA << 4 | bB << 6
// the vertex pairs in slot order: (0,0) (1,1) (2,2) (3,3) (0,1) (0,2) (0,3)
// (1,2) (1,3) (2,3)
__device__ __forceinline__ int pair_a(int p) { return p < 4 ? p : (p < 7 ? 0 : (p < 9 ? 1 : 2)); }
__device__ __forceinline__ int pair_b(int p) {
  return p < 4 ? p : (p == 4 ? 1 : (p == 5 || p == 7) ? 2 : 3);
}
struct SlotMeta {
  int a, b, c, d;
};
struct SlotTable {
  SlotMeta s[90];
};
constexpr int cst_cE0(int b) { return b == 2 ? 1 : (b == 1 ? -1 : 0); }
constexpr int cst_cE1(int b) { return b == 3 ? 1 : (b == 1 ? -1 : 0); }
constexpr SlotTable make_slot_table() {
  SlotTable t{};
  const int PA[10] = {0, 1, 2, 3, 0, 0, 0, 1, 1, 2}, PB[10] = {0, 1, 2, 3, 1, 2, 3, 2, 3, 3};
  for (int sl = 0; sl < 90; sl++) {
    const int pi = sl / 9, e = sl % 9, bA = PA[pi], bB = PB[pi], r = e / 3, c = e % 3;
    int I = 3 * bA + r, J = 3 * bB + c;
    if (I > J) {
      const int x = I;
      I = J;
      J = x;
    }
    const int bi = I / 3, bj = J / 3, ci = I % 3, cj = J % 3;
    int hdk = 0, hds = 0;  // sign 0: HD's entry is zero (ci == cj)
    if (ci != cj) {
      hdk = 3 - ci - cj;
      hds = ((cj - ci + 3) % 3 == 1) ? -1 : 1;
    }
    const int q00 = cst_cE0(bi) * cst_cE0(bj), q11 = cst_cE1(bi) * cst_cE1(bj);
    const int q01 = cst_cE0(bi) * cst_cE1(bj), q10 = cst_cE1(bi) * cst_cE0(bj);
    t.s[sl].a = I | (J << 4) | ((3 * pi + hdk) << 8) | ((hds + 1) << 14);
    t.s[sl].b = (3 * ci + cj) | ((3 * cj + ci) << 4) | ((q00 + 1) << 8) | ((q11 + 1) << 10) | ((q01 + 1) << 12) |
                ((q10 + 1) << 14);
    t.s[sl].c = (4 * bA + bB) | ((4 * bB + bA) << 4) | ((3 * r + c) << 8) | ((3 * c + r) << 12);
    t.s[sl].d = r | (c << 2) | (bA << 4) | (bB << 6);
  }
  return t;
}
__device__ const SlotTable kSlots = make_slot_table();

// the interior entry of a slot: u_I gD_J + w_I gS_J + c2 HD_IJ + c4 HS_IJ
__device__ __forceinline__ double plane_slot(const PlaneSetup &S, double c2, double c4, const SlotMeta &m) {
  const int I = m.a & 15, J = (m.a >> 4) & 15;
  const double hd = S.W[(m.a >> 8) & 63] * (double)(((m.a >> 14) & 3) - 1);
  const int ix = m.b & 15, ixt = (m.b >> 4) & 15;
  const double hs = (double)(((m.b >> 8) & 3) - 1) * S.h00[ix] + (double)(((m.b >> 10) & 3) - 1) * S.h11[ix] +
                    (double)(((m.b >> 12) & 3) - 1) * S.h01[ix] + (double)(((m.b >> 14) & 3) - 1) * S.h01[ixt];
  return S.u[I] * S.gD[J] + S.w[I] * S.gS[J] + c2 * hd + c4 * hs;
}

// Sixteen lanes per impact (two impacts per warp): every warp instruction of
// the per-impact setup serves two impacts, and twice as many impacts' loads
// are in flight per SM.  Group-local synchronisation only (the two halves of a
// warp may take different branches).
constexpr int GL = 32;                // lanes per impact
constexpr int GPW = 32 / GL;          // impacts per warp
constexpr int GROUPS = WARPS * GPW;   // impacts per block

__global__ void __launch_bounds__(32 * WARPS)
    k_imp_deriv(int n, const int4 *__restrict__ imp, const double4 *__restrict__ xc,
                const int4 *__restrict__ ci, const double4 *__restrict__ cd, double kpen,
                const int *__restrict__ pos, double *__restrict__ rec, double *__restrict__ frc) {
  __shared__ PlaneSetup sP[GROUPS];
  __shared__ LineSetup sL[GROUPS];
  __shared__ double sx[GROUPS][12];
  __shared__ double sfd[GROUPS][3];
  __shared__ int sPos[GROUPS][16];
  const int lane = threadIdx.x & 31;
  const int gi = threadIdx.x / GL, gl = threadIdx.x % GL;  // group in the block, lane in the group
  const unsigned gmask = (GL == 32) ? 0xffffffffu : (((1u << GL) - 1u) << (lane & ~(GL - 1)));
  const int u = blockIdx.x * GROUPS + gi;
  if (u >= n) return;  // uniform per group
  const int *P = pos + 16 * (size_t)u;
  const int4 c = ci[u];
  for (int l = gl; l < 16; l += GL) sPos[gi][l] = P[l];
  if (c.x < 0) {  // no response: zero records, zero forces
    for (int e = gl; e < 16 * ICF_IMP_REC; e += GL) {
      const int q = P[e / ICF_IMP_REC];
      if (q >= 0) rec[ICF_IMP_REC * (size_t)q + e % ICF_IMP_REC] = 0.0;
    }
    for (int l = gl; l < 12; l += GL) frc[12 * (size_t)u + l] = 0.0;
    return;
  }
  const double4 cl = cd[u];
  const int4 id = imp[u];
  if (gl < 4) {
    const int nd = gl == 0 ? id.x : gl == 1 ? id.y : gl == 2 ? id.z : id.w;
    const double4 p = xc[nd];
    sx[gi][3 * gl] = p.x;
    sx[gi][3 * gl + 1] = p.y;
    sx[gi][3 * gl + 2] = p.z;
  }
  __syncwarp(gmask);
  const double *x = sx[gi];
  const double hk = kpen * 0.5;
  const int kind = c.x;
  double c2 = 0, c4 = 0;  // interior: the scalars of HD and HS
  if (kind == 1) {  // vertex: d2 = |p - x_b|^2
    if (gl < 3) sfd[gi][gl] = 2 * (x[gl] - x[3 * c.z + gl]);
  } else if (kind == 2) {  // edge (ia nearer, ib)
    const int ia = c.y, ib = c.z;
    LineSetup &L = sL[gi];
    if (gl == 0) {
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
        sfd[gi][k] = L.f1d[k] + (L.g * L.f2d[k] - L.f2 * L.gd[k]) / L.f2sq;
    }
  } else {  // interior: d2 = D^2 / S
    PlaneSetup &S = sP[gi];
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
    for (int l = gl; l < 12; l += GL) {
      const int b = l / 3, k = l % 3;
      const double gd = cA(b) * pick3(N, k) + cE0(b) * pick3(e1xa, k) + cE1(b) * pick3(axe0, k);
      const double gs = 2.0 * (cE0(b) * pick3(e1xN, k) + cE1(b) * pick3(Nxe0, k));
      S.gD[l] = gd;
      S.gS[l] = gs;
      S.u[l] = c1 * gd + c3 * gs;
      S.w[l] = c3 * gd + c5 * gs;
    }
    // HS blocks, S = |e0|^2 |e1|^2 - (e0.e1)^2
    {
      const double e00 = e0[0] * e0[0] + e0[1] * e0[1] + e0[2] * e0[2];
      const double e11 = e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2];
      const double e01 = e0[0] * e1[0] + e0[1] * e1[1] + e0[2] * e1[2];
      for (int l = gl; l < 9; l += GL) {
        const int r = l / 3, q = l % 3;
        const double dl = r == q ? 1.0 : 0.0;
        const double e0r = pick3(e0, r), e0q = pick3(e0, q), e1r = pick3(e1, r), e1q = pick3(e1, q);
        S.h00[l] = 2.0 * (e11 * dl - e1r * e1q);
        S.h11[l] = 2.0 * (e00 * dl - e0r * e0q);
        S.h01[l] = 4.0 * e0r * e1q - 2.0 * e1r * e0q - 2.0 * e01 * dl;
      }
    }
    // W per vertex-block pair (bi <= bj, the slots' pairs): D is trilinear in
    // (a, e0, e1), so HD's block (bi, bj) is [W]x, W = -e1 (ai pj0 - pi0 aj) + e0 (ai pj1 - pi1 aj)
    // - a (pi0 pj1 - pi1 pj0)
    for (int l = gl; l < 30; l += GL) {
      const int pr = l / 3, k = l % 3, bi = pair_a(pr), bj = pair_b(pr);
      const double ai = cA(bi), aj = cA(bj), pi0 = cE0(bi), pj0 = cE0(bj), pi1 = cE1(bi), pj1 = cE1(bj);
      const double al = ai * pj0 - pi0 * aj, be = ai * pj1 - pi1 * aj, ga = pi0 * pj1 - pi1 * pj0;
      S.W[l] = -pick3(e1, k) * al + pick3(e0, k) * be - pick3(a, k) * ga;
    }
    // d(d2)/dp = 2 D N / S
    if (gl < 3) sfd[gi][gl] = c2 * pick3(N, gl);
  }
  __syncwarp(gmask);
  // one lane per record entry: pair (bA, bB), entry (r, c); a lane's entries
  // are computed first and stored after, so that their shared-memory reads
  // overlap
  constexpr int NS = (90 + GL - 1) / GL;
  double val[NS];
  long long dst[NS];
#pragma unroll
  for (int k = 0; k < NS; k++) {
    const int sl = gl + GL * k;
    val[k] = 0.0;
    dst[k] = -1;
    if (sl < 90) {
      const SlotMeta m = kSlots.s[sl];
      const int I = m.a & 15, J = (m.a >> 4) & 15;
      double v = 0;
      if (kind == 1) {
        const int vb = c.z, bI = I / 3, bJ = J / 3;
        if (I % 3 == J % 3 && (bI == 0 || bI == vb) && (bJ == 0 || bJ == vb)) v = (bI == bJ) ? 2.0 : -2.0;
      } else if (kind == 2) {
        const int ia = c.y, ib = c.z, bI = I / 3, bJ = J / 3;
        const int pI = bI == 0 ? 0 : (bI == ia ? 1 : (bI == ib ? 2 : -1));
        const int pJ = bJ == 0 ? 0 : (bJ == ia ? 1 : (bJ == ib ? 2 : -1));
        if (pI >= 0 && pJ >= 0) v = line_entry(sL[gi], 3 * pI + I % 3, 3 * pJ + J % 3);
      } else {
        v = plane_slot(sP[gi], c2, c4, m);
      }
      val[k] = kpen * v / 2;
      // the code of the pair, taken either way round (none: an anchored vertex)
      const int q = sPos[gi][m.c & 15];
      if (q >= 0) {
        dst[k] = ICF_IMP_REC * (long long)q + ((m.c >> 8) & 15);
      } else if ((m.c & 15) != ((m.c >> 4) & 15)) {
        const int q2 = sPos[gi][(m.c >> 4) & 15];
        if (q2 >= 0) dst[k] = ICF_IMP_REC * (long long)q2 + ((m.c >> 12) & 15);
      }
    }
  }
#pragma unroll
  for (int k = 0; k < NS; k++)
    if (dst[k] >= 0) rec[dst[k]] = val[k];
  // vertex forces (-F, w0 F, w1 F, w2 F), F = k/2 d(d2)/dp, w = (1-s-t, s, t)
  // (collision_response.h:89-109): into the force record, and as the rhs of
  // the vertex's diagonal code; off-diagonal codes carry no rhs
  for (int l = gl; l < 12; l += GL) {
    const double s = cl.x, t = cl.y;
    const int comp = l % 3, blk = l / 3;
    const double F = hk * sfd[gi][comp];
    const double f = blk == 0 ? -F : (blk == 1 ? (1 - (s + t)) : (blk == 2 ? s : t)) * F;
    frc[12 * (size_t)u + l] = f;
    const int q = sPos[gi][5 * blk];
    if (q >= 0) rec[ICF_IMP_REC * (size_t)q + 9 + comp] = f;
  }
  for (int pr = gl; pr < 16; pr += GL) {
    const int q = sPos[gi][pr];
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
  k_imp_deriv<<<icf_blocks(ctx->n_imp, GROUPS), 32 * WARPS, 0, stream>>>(
      ctx->n_imp, ctx->d_imp, xc, cls_i, cls_d, ctx->prm.penaltyK, ctx->d_imp_pos, ks,
      icf_imp_forces(ks, ctx->n_imp));
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}
