// icf_contact_deriv.cu -- penalty response of the impacts, one thread per impact.
//
// kCollisionResponseForce (collision_response.h:38-127): whether the impact
// responds (a vertex off the anchors, distance above DistanceEpsilon, :47-51
// and :91), then the gradient and Hessian of the squared point-triangle
// distance d2(x), x = (p, v0, v1, v2), in its Voronoi region (pt_classify,
// icf_ptri.cuh):
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
// HS follows from S = |e0|^2 |e1|^2 - (e0.e1)^2.  About 10 operations per
// entry instead of some 200; the two forms agree to rounding (1e-14 of the
// largest entry on random interior cases).
//
// One thread computes an impact's whole response.  The ten vertex pairs
// (p, v0, v1, v2 taken two at a time, diagonal pairs included) and the
// entries of their 3x3 blocks are unrolled at compile time, so every
// coefficient that depends only on the pair (the +-1/0 weights of a, e0, e1
// in each vertex's gradient, HD's cross-product vector, HS's terms) folds
// into the instruction stream: no tables, no shared memory, no index
// arithmetic per entry.  K = k/2 d2'' goes to the record of the pair's
// contribution code at its position in the slot-sorted list (icf_internal.cuh,
// ICF_IMP_REC): the block in the code's orientation, then, on a diagonal code,
// the vertex's rhs from (-F, w0 F, w1 F, w2 F), F = k/2 d(d2)/dp,
// w = (1-s-t, s, t), else zeros; a record is three 32-byte stores (FP32-mixed:
// the block in FP32, then the rhs, two 32-byte stores).  A diagonal
// block's lower entries are its upper ones, so it is symmetric bit for bit.
// The four vertex forces also go to a per-impact force record (node forces).
#include "icf_internal.cuh"
#include "icf_ptri.cuh"
#include "icf_tet.cuh"

// This file is compiled with -fmad=false (pt_classify's region decision must
// round every operation on its own); the Hessian arithmetic is unfused too.

namespace {

#ifndef IMP_TPB
#define IMP_TPB 128
#endif
#ifndef IMP_MINB
#define IMP_MINB 1
#endif
constexpr int TPB = IMP_TPB;

// coefficients of vertex block b (p, v0, v1, v2) in a = p - v0,
// e0 = v1 - v0, e1 = v2 - v0 (compile-time after unrolling)
__host__ __device__ constexpr int cA(int b) { return b == 0 ? 1 : (b == 1 ? -1 : 0); }
__host__ __device__ constexpr int cE0(int b) { return b == 2 ? 1 : (b == 1 ? -1 : 0); }
__host__ __device__ constexpr int cE1(int b) { return b == 3 ? 1 : (b == 1 ? -1 : 0); }

__device__ __forceinline__ void st4(double *p, double a, double b, double c, double d) {
  asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(a), "d"(b), "d"(c), "d"(d) : "memory");
}

// Two FP32 values in one 64-bit word: a in the low half, b in the high half.
__device__ __forceinline__ double pack2(double a, double b) {
  return __hiloint2double(__float_as_int((float)b), __float_as_int((float)a));
}

// The record of vertex pair (bA, bB): to the code (bA, bB) if there is one,
// else the block transposed to the code (bB, bA) (none: an anchored vertex).
// Records start at 96-byte multiples, so each third is 32-byte aligned.
// FP64: the block, then the rhs, in three 32-byte stores.  FP32-mixed: the
// block rounded to FP32 (two values per 64-bit word), then the rhs in FP64,
// in the first two 32-byte sectors of the record's slot.
template <bool MIXED>
__device__ __forceinline__ void put_record(double *__restrict__ rec, int q, int qt, const double B[9], double f0,
                                           double f1, double f2) {
  const bool fw = q >= 0;
  if (!fw && qt < 0) return;
  double *o = rec + ICF_IMP_REC * (size_t)(fw ? q : qt);
  // the entries in the code's orientation
  const double b0 = B[0], b1 = fw ? B[1] : B[3], b2 = fw ? B[2] : B[6], b3 = fw ? B[3] : B[1], b4 = B[4];
  const double b5 = fw ? B[5] : B[7], b6 = fw ? B[6] : B[2], b7 = fw ? B[7] : B[5], b8 = B[8];
  if (MIXED) {
    st4(o, pack2(b0, b1), pack2(b2, b3), pack2(b4, b5), pack2(b6, b7));
    st4(o + 4, pack2(b8, 0.0), f0, f1, f2);
  } else {
    st4(o, b0, b1, b2, b3);
    st4(o + 4, b4, b5, b6, b7);
    st4(o + 8, b8, f0, f1, f2);
  }
}

// Interior region: everything an entry needs, per impact.
struct Plane {
  double a[3], e0[3], e1[3];
  double gD[12], gS[12];
  double c1, c2, c3, c4, c5;
  double e00, e11, e01;
};

// HS's 3x3 blocks over (e0, e0), (e1, e1), (e0, e1) at (r, q)
__device__ __forceinline__ double hs00(const Plane &P, int r, int q) {
  return 2.0 * ((r == q ? P.e11 : 0.0) - P.e1[r] * P.e1[q]);
}
__device__ __forceinline__ double hs11(const Plane &P, int r, int q) {
  return 2.0 * ((r == q ? P.e00 : 0.0) - P.e0[r] * P.e0[q]);
}
__device__ __forceinline__ double hs01(const Plane &P, int r, int q) {
  return 4.0 * P.e0[r] * P.e1[q] - 2.0 * P.e1[r] * P.e0[q] - (r == q ? 2.0 * P.e01 : 0.0);
}

// block (bi, bj) of the interior Hessian (bi <= bj), row-major
template <int bi, int bj>
__device__ __forceinline__ void block(const Plane &P, double B[9]) {
  // HD's block is [W]x, W = -e1 al + e0 be - a ga (D trilinear in a, e0, e1)
  constexpr int al = cA(bi) * cE0(bj) - cE0(bi) * cA(bj);
  constexpr int be = cA(bi) * cE1(bj) - cE1(bi) * cA(bj);
  constexpr int ga = cE0(bi) * cE1(bj) - cE1(bi) * cE0(bj);
  constexpr int q00 = cE0(bi) * cE0(bj), q11 = cE1(bi) * cE1(bj);
  constexpr int q01 = cE0(bi) * cE1(bj), q10 = cE1(bi) * cE0(bj);
  double W[3];
#pragma unroll
  for (int k = 0; k < 3; k++) W[k] = -P.e1[k] * (double)al + P.e0[k] * (double)be - P.a[k] * (double)ga;
#pragma unroll
  for (int r = 0; r < 3; r++) {
    const int I = 3 * bi + r;
    const double u = P.c1 * P.gD[I] + P.c3 * P.gS[I];
    const double w = P.c3 * P.gD[I] + P.c5 * P.gS[I];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      if (bi == bj && c < r) {
        B[3 * r + c] = B[3 * c + r];
        continue;
      }
      const int J = 3 * bj + c;
      double hd = 0.0;
      if (r != c) {
        const int k = 3 - r - c;
        hd = ((c - r + 3) % 3 == 1) ? -W[k] : W[k];
      }
      double hs = 0.0;
      if (q00) hs += (double)q00 * hs00(P, r, c);
      if (q11) hs += (double)q11 * hs11(P, r, c);
      if (q01) hs += (double)q01 * hs01(P, r, c);
      if (q10) hs += (double)q10 * hs01(P, c, r);
      B[3 * r + c] = u * P.gD[J] + w * P.gS[J] + P.c2 * hd + P.c4 * hs;
    }
  }
}

// Edge region: d2 = f1 - g / f2 over y = (p, q1, q2), spread over the four
// vertex blocks (q1 = block ia, q2 = block ib, the fourth block zero).
struct Line {
  double spd[12], f2d[12], gd[12];
  double sp, g, if2, if2sq, if2cu;
  int m[4];  // block -> 0 (p), 1 (q1), 2 (q2), -1 (none)
};

template <int bi, int bj>
__device__ __forceinline__ void block(const Line &L, double B[9]) {
  const int pI = L.m[bi], pJ = L.m[bj];
  if (pI < 0 || pJ < 0) {
#pragma unroll
    for (int e = 0; e < 9; e++) B[e] = 0.0;
    return;
  }
  // second derivatives of sp, f1, f2 between the blocks (times the identity)
  const double spdd = (pI == 1 && pJ == 1) ? -2.0 : ((pI + pJ == 2 && pI != pJ) ? -1.0 : (pI != pJ ? 1.0 : 0.0));
  const double f1dd = (pI != 2 && pJ != 2) ? (pI == pJ ? 2.0 : -2.0) : 0.0;
  const double f2dd = (pI != 0 && pJ != 0) ? (pI == pJ ? 2.0 : -2.0) : 0.0;
#pragma unroll
  for (int r = 0; r < 3; r++) {
    const int I = 3 * bi + r;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      if (bi == bj && c < r) {
        B[3 * r + c] = B[3 * c + r];
        continue;
      }
      const int J = 3 * bj + c;
      const double dl = r == c ? 1.0 : 0.0;
      const double gdd = 2 * (L.spd[I] * L.spd[J] + L.sp * spdd * dl);
      const double t1 = -2 * L.g * L.f2d[I] * L.f2d[J] * L.if2cu;
      const double t2 = (L.gd[I] * L.f2d[J] + L.gd[J] * L.f2d[I]) * L.if2sq;
      const double t4 = L.g * f2dd * dl * L.if2sq;
      const double t5 = -gdd * L.if2;
      B[3 * r + c] = t1 + t2 + f1dd * dl + t4 + t5;
    }
  }
}

// Vertex region, d2 = |p - x_vb|^2: 2 I on (p, p) and (vb, vb), -2 I on (p, vb).
struct Vertex {
  int vb;
};
template <int bi, int bj>
__device__ __forceinline__ void block(const Vertex &V, double B[9]) {
  const bool on = (bi == 0 || bi == V.vb) && (bj == 0 || bj == V.vb);
  const double d = on ? (bi == bj ? 2.0 : -2.0) : 0.0;
#pragma unroll
  for (int e = 0; e < 9; e++) B[e] = (e % 4 == 0) ? d : 0.0;
}

template <int bi, int bj, bool MIXED, class Region>
__device__ __forceinline__ void emit_pair(const Region &R, double hk, const int pos[16], const double frc[12],
                                          double *__restrict__ rec) {
  double B[9];
  block<bi, bj>(R, B);
#pragma unroll
  for (int e = 0; e < 9; e++) B[e] *= hk;  // K = k/2 d2''
  if (bi == bj) put_record<MIXED>(rec, pos[5 * bi], -1, B, frc[3 * bi], frc[3 * bi + 1], frc[3 * bi + 2]);
  else put_record<MIXED>(rec, pos[4 * bi + bj], pos[4 * bj + bi], B, 0.0, 0.0, 0.0);
}

// The impact's vertex forces (-F, w0 F, w1 F, w2 F), F = k/2 d(d2)/dp,
// w = (1-s-t, s, t) (collision_response.h:89-109), to its force record, then
// the ten records.
template <bool MIXED, class Region>
__device__ __forceinline__ void respond(const Region &R, const double fd[3], double hk, double s, double t,
                                        const int pos[16], double *__restrict__ fo, double *__restrict__ rec) {
  double frc[12];
  const double w0 = 1 - (s + t);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const double F = hk * fd[k];
    frc[k] = -F;
    frc[3 + k] = w0 * F;
    frc[6 + k] = s * F;
    frc[9 + k] = t * F;
  }
#pragma unroll
  for (int k = 0; k < 12; k += 4) st4(fo + k, frc[k], frc[k + 1], frc[k + 2], frc[k + 3]);
  emit_pair<0, 0, MIXED>(R, hk, pos, frc, rec);
  emit_pair<1, 1, MIXED>(R, hk, pos, frc, rec);
  emit_pair<2, 2, MIXED>(R, hk, pos, frc, rec);
  emit_pair<3, 3, MIXED>(R, hk, pos, frc, rec);
  emit_pair<0, 1, MIXED>(R, hk, pos, frc, rec);
  emit_pair<0, 2, MIXED>(R, hk, pos, frc, rec);
  emit_pair<0, 3, MIXED>(R, hk, pos, frc, rec);
  emit_pair<1, 2, MIXED>(R, hk, pos, frc, rec);
  emit_pair<1, 3, MIXED>(R, hk, pos, frc, rec);
  emit_pair<2, 3, MIXED>(R, hk, pos, frc, rec);
}

template <bool MIXED>
__global__ void __launch_bounds__(TPB, IMP_MINB)
    k_imp_deriv(int n, const int4 *__restrict__ imp, const int *__restrict__ alt, const double4 *__restrict__ xc,
                double eps2, double kpen, const int *__restrict__ pos16, double *__restrict__ rec,
                double *__restrict__ frc_out, int *__restrict__ counts) {
  const int u = blockIdx.x * TPB + threadIdx.x;
  if (u >= n) return;
  int pos[16];
  {
    const int4 *P4 = reinterpret_cast<const int4 *>(pos16 + 16 * (size_t)u);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int4 v = __ldg(P4 + k);
      pos[4 * k] = v.x;
      pos[4 * k + 1] = v.y;
      pos[4 * k + 2] = v.z;
      pos[4 * k + 3] = v.w;
    }
  }
  const int4 id = __ldg(imp + u);
  const int nd[4] = {id.x, id.y, id.z, id.w};
  bool any_active = false, valid = true;
#pragma unroll
  for (int b = 0; b < 4; b++) {
    valid &= nd[b] >= 0;
    any_active |= (nd[b] >= 0 && __ldg(alt + nd[b]) >= 0);
  }
  double x[12];
  pt_cls cl;
  cl.kind = -1;
  if (valid && any_active) {
#pragma unroll
    for (int b = 0; b < 4; b++) ld_node(xc, nd[b], x + 3 * b);
    cl = pt_classify(x);
    if (!(cl.dsq > eps2)) cl.kind = -1;  // within DistanceEpsilon: no response
  }
  // the impacts that respond, one atomic per group of converged lanes (the
  // same mask for the vote and the choice of the lane that adds)
  const unsigned am = __activemask();
  const unsigned act = __ballot_sync(am, cl.kind >= 0);
  if ((int)(threadIdx.x & 31) == __ffs(am) - 1 && act) atomicAdd(counts + 3, __popc(act));
  double *fo = frc_out + 12 * (size_t)u;
  if (cl.kind < 0) {  // no response: zero records, zero forces
#pragma unroll
    for (int k = 0; k < 16; k++)
      if (pos[k] >= 0) {
        double *o = rec + ICF_IMP_REC * (size_t)pos[k];
        st4(o, 0.0, 0.0, 0.0, 0.0);
        st4(o + 4, 0.0, 0.0, 0.0, 0.0);
        if (!MIXED) st4(o + 8, 0.0, 0.0, 0.0, 0.0);
      }
#pragma unroll
    for (int k = 0; k < 12; k += 4) st4(fo + k, 0.0, 0.0, 0.0, 0.0);
    return;
  }
  const int4 c = make_int4(cl.kind, cl.ia, cl.ib, 0);
  const double2 st = make_double2(cl.s, cl.t);
  const double hk = kpen * 0.5;
  const int kind = c.x;
  double fd[3];  // d(d2)/dp
  if (kind == 1) {  // vertex: d2 = |p - x_b|^2
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const double xb = c.z == 1 ? x[3 + k] : (c.z == 2 ? x[6 + k] : x[9 + k]);
      fd[k] = 2 * (x[k] - xb);
    }
    respond<MIXED>(Vertex{c.z}, fd, hk, st.x, st.y, pos, fo, rec);
  } else if (kind == 2) {  // edge (ia nearer, ib)
    const int ia = c.y, ib = c.z;
    Line L;
    double Q1[3], Q2[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      Q1[k] = ia == 1 ? x[3 + k] : (ia == 2 ? x[6 + k] : x[9 + k]);
      Q2[k] = ib == 1 ? x[3 + k] : (ib == 2 ? x[6 + k] : x[9 + k]);
    }
    double sp = 0, f2 = 0, spd_p[3], spd_1[3], spd_2[3], f2d_1[3], f2d_2[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const double a = Q1[k] - x[k], b = Q2[k] - Q1[k];
      spd_p[k] = Q1[k] - Q2[k];
      spd_1[k] = x[k] - 2 * Q1[k] + Q2[k];
      spd_2[k] = Q1[k] - x[k];
      sp += a * b;
      f2 += b * b;
      f2d_1[k] = -(2 * b);
      f2d_2[k] = 2 * b;
    }
    L.sp = sp;
    L.g = sp * sp;
    L.if2 = 1.0 / f2;
    L.if2sq = L.if2 * L.if2;
    L.if2cu = L.if2sq * L.if2;
    L.m[0] = 0;
#pragma unroll
    for (int b = 1; b < 4; b++) L.m[b] = b == ia ? 1 : (b == ib ? 2 : -1);
#pragma unroll
    for (int b = 0; b < 4; b++)
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const int mb = L.m[b];
        L.spd[3 * b + k] = mb == 0 ? spd_p[k] : (mb == 1 ? spd_1[k] : (mb == 2 ? spd_2[k] : 0.0));
        L.f2d[3 * b + k] = mb == 1 ? f2d_1[k] : (mb == 2 ? f2d_2[k] : 0.0);
        L.gd[3 * b + k] = 2 * sp * L.spd[3 * b + k];
      }
    // f1 - g / f2 differentiated in p: f1' = -2 (q1 - p), f2' = 0
#pragma unroll
    for (int k = 0; k < 3; k++) fd[k] = -(2 * (Q1[k] - x[k])) - L.gd[k] * L.if2;
    respond<MIXED>(L, fd, hk, st.x, st.y, pos, fo, rec);
  } else {  // interior: d2 = D^2 / S
    Plane P;
    double N[3], e1xa[3], axe0[3], e1xN[3], Nxe0[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      P.a[k] = x[k] - x[3 + k];
      P.e0[k] = x[6 + k] - x[3 + k];
      P.e1[k] = x[9 + k] - x[3 + k];
    }
#define CROSS(o, u_, v_)                \
  o[0] = u_[1] * v_[2] - u_[2] * v_[1]; \
  o[1] = u_[2] * v_[0] - u_[0] * v_[2]; \
  o[2] = u_[0] * v_[1] - u_[1] * v_[0];
    CROSS(N, P.e0, P.e1)
    CROSS(e1xa, P.e1, P.a)
    CROSS(axe0, P.a, P.e0)
    CROSS(e1xN, P.e1, N)
    CROSS(Nxe0, N, P.e0)
#undef CROSS
    const double D = P.a[0] * N[0] + P.a[1] * N[1] + P.a[2] * N[2];
    const double Sv = N[0] * N[0] + N[1] * N[1] + N[2] * N[2];
    const double iS = 1.0 / Sv;
    P.c1 = 2.0 * iS;
    P.c3 = -2.0 * D * iS * iS;
    P.c5 = 2.0 * D * D * iS * iS * iS;
    P.c2 = 2.0 * D * iS;
    P.c4 = -D * D * iS * iS;
#pragma unroll
    for (int b = 0; b < 4; b++)
#pragma unroll
      for (int k = 0; k < 3; k++) {
        P.gD[3 * b + k] = (double)cA(b) * N[k] + (double)cE0(b) * e1xa[k] + (double)cE1(b) * axe0[k];
        P.gS[3 * b + k] = 2.0 * ((double)cE0(b) * e1xN[k] + (double)cE1(b) * Nxe0[k]);
      }
    P.e00 = P.e0[0] * P.e0[0] + P.e0[1] * P.e0[1] + P.e0[2] * P.e0[2];
    P.e11 = P.e1[0] * P.e1[0] + P.e1[1] * P.e1[1] + P.e1[2] * P.e1[2];
    P.e01 = P.e0[0] * P.e1[0] + P.e0[1] * P.e1[1] + P.e0[2] * P.e1[2];
    // d(d2)/dp = 2 D N / S
#pragma unroll
    for (int k = 0; k < 3; k++) fd[k] = P.c2 * N[k];
    respond<MIXED>(P, fd, hk, st.x, st.y, pos, fo, rec);
  }
}

}  // namespace

int icf_launch_imp_deriv(icf_ctx *ctx, cudaStream_t stream) {
  return icf_launch_imp_deriv_bufs(ctx, ctx->d_xc, ctx->d_ks, stream);
}

// Derivative kernel with caller-chosen buffers (the allocation-free entry
// point passes its own staging).
int icf_launch_imp_deriv_bufs(icf_ctx *ctx, const double4 *xc, double *ks, cudaStream_t stream) {
  const double eps2 = ctx->prm.DistanceEpsilon * ctx->prm.DistanceEpsilon;
  auto kern = ctx->precision == ICF_FP32_MIXED ? k_imp_deriv<true> : k_imp_deriv<false>;
  kern<<<icf_blocks(ctx->n_imp, TPB), TPB, 0, stream>>>(ctx->n_imp, ctx->d_imp, ctx->d_alt, xc, eps2,
                                                                ctx->prm.penaltyK, ctx->d_imp_pos, ks,
                                                                icf_imp_forces(ks, ctx->n_imp), ctx->d_counts);
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}
