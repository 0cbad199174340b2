// icf_assembly.cu -- per-unit kernels and the atomic-free BCSR gather.
//
// One assembly (icf_launch_assembly) is:
//   k_tet_unit    one thread per tetrahedron: corotational force, rotated
//                 shape-function gradients and the Newmark rhs of each vertex
//                 (element_kernels2.h:19-159 and :195-263) -> tet staging
//   k_cz_gp       three threads per cohesive zone, one per Gauss point:
//                 mid-plane frame, PPR law, then the Gauss points combine into
//                 the CZ staging, tentative damage state and flags
//                 (cz_kernels.h:210-434)
//   k_imp_*       impacts (icf_contact.cu, icf_contact_deriv.cu)
//   k_gather_*    (icf_gather.cu) the lanes that own a BCSR block sum the
//                 contributions listed for it in the pattern's sliced-ELL
//                 lists and write it once (and the rhs row of a diagonal
//                 block, with the NaN/Inf check of the row)
//   k_imp_add     adds impact contributions to the blocks they touch
// Each block is summed in a fixed order and written once, so the result is
// bit-reproducible; the reference's CAS-loop atomics (atomic_add.h:1-13) have
// no counterpart.
#include <vector>

#include "icf_internal.cuh"
#include "icf_ppr.cuh"
#include "icf_tet.cuh"

namespace {

// One thread per tetrahedron.  Each warp's 32 records (8 KB) are staged in
// shared memory (rows padded to 272 B, so both the row-wise writes and the
// column-wise reads are free of bank conflicts) and stored as 512 B
// contiguous chunks per instruction.
//
// FP32-mixed (MIXED): the rotation, the force and the rhs stay FP64; the
// rotated gradients and the volume, which are all the Hessian blocks are
// built from, are rounded to FP32.  The staging then holds the rhs records
// compactly, es[4e + a] = {rhs_a, 0}, followed by the FP32 records
// es32[4e + a] = {h_a, V} with es32 = (float4 *)(es + 4 ne): 192 B per tet in
// the same buffer.
template <int MINB, bool MIXED>
__global__ void __launch_bounds__(128, MINB)
    k_tet_unit(int ne, const int4 *__restrict__ elem,
               const double4 *__restrict__ x0, const double4 *__restrict__ xc,
               const double2 *__restrict__ va, icf_dprm P,
               double4 *__restrict__ es) {
  __shared__ double2 sbuf[4][32][17];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const long long base = (long long)blockIdx.x * blockDim.x + 32 * w;
  if (base >= ne) return;
  const int e = (int)base + lane;
  if (e < ne) tet_record<MIXED>(e, elem, x0, xc, va, P, sbuf[w][lane]);
  __syncwarp();
  const long long nrec = (ne - base) < 32 ? (ne - base) : 32;
  if (!MIXED) {
    double2 *o = reinterpret_cast<double2 *>(es) + 16 * base;
#pragma unroll 4
    for (int k = 0; k < 16; k++) {
      const int idx = 32 * k + lane;
      if (idx < 16 * nrec) o[idx] = sbuf[w][idx >> 4][idx & 15];
    }
  } else {
    double2 *o = reinterpret_cast<double2 *>(es) + 8 * base;
#pragma unroll 4
    for (int k = 0; k < 8; k++) {
      const int idx = 32 * k + lane;
      if (idx < 8 * nrec) o[idx] = sbuf[w][idx >> 3][idx & 7];
    }
    float4 *oh = reinterpret_cast<float4 *>(es + 4 * (size_t)ne) + 4 * base;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int idx = 32 * k + lane;
      if (idx < 4 * nrec) oh[idx] = *reinterpret_cast<const float4 *>(&sbuf[w][idx >> 2][8 + (idx & 3)]);
    }
  }
}

// ---- cohesive zones -------------------------------------------------------------
// Geometry up to the Gauss-point openings is evaluated with separately
// rounded products and sums (the __d*_rn intrinsics are never fused), so the
// openings that drive the law's branch decisions are the same numbers the
// checker computes.  Everything after the law may use fused multiply-adds.
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// CZRotationMatrix (cz_kernels9/matrix_math.h:15-68).
__device__ __forceinline__ void cz_frame(const double m0[3], const double m1[3],
                                         const double m2[3], double R[3][3],
                                         double &aJ) {
  double p1[3], p2[3], n[3], r[3];
  for (int k = 0; k < 3; k++) {
    p1[k] = sub(m1[k], m0[k]);
    p2[k] = sub(m0[k], m2[k]);
  }
  // the reference's operation order and rounding (no contraction): the
  // opening is a difference of nearly equal rotated coordinates, so a
  // rounding change in R moves it by far more than its own size at small
  // openings
  const double l1 = sqrt(add(add(mul(p1[0], p1[0]), mul(p1[1], p1[1])), mul(p1[2], p1[2])));
  for (int k = 0; k < 3; k++) R[0][k] = p1[k] / l1;
  n[0] = add(mul(-p1[2], p2[1]), mul(p1[1], p2[2]));
  n[1] = sub(mul(p1[2], p2[0]), mul(p1[0], p2[2]));
  n[2] = add(mul(-p1[1], p2[0]), mul(p1[0], p2[1]));
  double ln = sqrt(add(add(mul(n[0], n[0]), mul(n[1], n[1])), mul(n[2], n[2])));
  aJ = ln / 2;
  for (int k = 0; k < 3; k++) {
    n[k] = n[k] / ln;
    R[2][k] = n[k];
    p1[k] = p1[k] / l1;
  }
  r[0] = add(mul(-n[2], p1[1]), mul(n[1], p1[2]));
  r[1] = sub(mul(n[2], p1[0]), mul(n[0], p1[2]));
  r[2] = add(mul(-n[1], p1[0]), mul(n[0], p1[1]));
  ln = sqrt(add(add(mul(r[0], r[0]), mul(r[1], r[1])), mul(r[2], r[2])));
  for (int k = 0; k < 3; k++) R[1][k] = r[k] / ln;
}

// Staging of one CZ (ICF_CZ_STAGE doubles).  With s_a = +sf[a][gp] for the
// first face's vertices (a < 3) and -sf[a-3][gp] for the second's, the
// reference's B^T T_d B (cz_kernels.h:366-401) gives the block
//   Keff_ab = sum_gp s_a s_b Q_gp,   Q_gp = (aJ/3) R^T T_d R
// and the rhs rhs_a = -sum_gp s_a (aJ/3) R^T T (:343-364).  Both depend on a
// and b only through a mod 3, b mod 3 and the face signs, so the record holds
//   Kt[i][j] = sum_gp sf[i][gp] sf[j][gp] Q_gp   (i <= j, symmetric 3x3: 6)
//   rt[i]    = sum_gp sf[i][gp] (aJ/3) R^T T_gp  (3)
// i.e. 36 + 9 doubles.
//
// Three threads per CZ, one per Gauss point: each evaluates the frame, its
// opening and the law; the three combine through shared memory in Gauss point
// order 0, 1, 2 (the reference's accumulation order).
constexpr int CZ_PER_BLOCK = 32;
// FP32-mixed (MIXED): geometry, law and tractions stay FP64 (the PPR law,
// including its softening branch near separation, is FP64 throughout); the
// Gauss-point tangents Q and their combination into the 3x3 blocks Kt are
// FP32.  The staging then holds rt compactly, cs[12c + 0..8] (FP64), followed
// by the FP32 blocks cs32[36c + 0..35] with cs32 = (float *)(cs + 12 nc):
// 240 B per CZ in the same buffer.
template <bool MIXED, int MINB, bool EXACT = false>
__global__ void __launch_bounds__(3 * CZ_PER_BLOCK, MINB)
    k_cz_gp(int nc, const int *__restrict__ cz, const double4 *__restrict__ xc,
            const double *__restrict__ czs, const int *__restrict__ czfail,
            const double4 *__restrict__ czprm, const double *__restrict__ hist, icf_dprm P, icf_law_c LC,
            double *__restrict__ cs, double *__restrict__ cztent, int *__restrict__ czflags,
            double *__restrict__ czavg, int *__restrict__ counts) {
  __shared__ double sQ[3 * CZ_PER_BLOCK][6];
  __shared__ double sTw[3 * CZ_PER_BLOCK][3];
  __shared__ double sAv[3 * CZ_PER_BLOCK][4];
  __shared__ double sPT[3 * CZ_PER_BLOCK][2];
  __shared__ int sFl[3 * CZ_PER_BLOCK];
  __shared__ double sOut[CZ_PER_BLOCK * ICF_CZ_STAGE];
  __shared__ double sD[CZ_PER_BLOCK][9];   // per CZ: (R x_n - R x_{n+3})[k] at 3 n + k
  __shared__ double sRJ[CZ_PER_BLOCK][10]; // per CZ: R (row-major), aJ
  const int t = threadIdx.x;
  // per CZ, once (the first warp, one CZ per lane): node positions, the
  // mid-plane, its frame and the rotated face differences (:243-290)
  if (t < CZ_PER_BLOCK) {
    const int cc = blockIdx.x * CZ_PER_BLOCK + t;
    if (cc < nc && __ldg(czfail + cc) == 0) {
      const int4 i0 = __ldg(reinterpret_cast<const int4 *>(cz) + 2 * cc);
      const int2 i1 = __ldg(reinterpret_cast<const int2 *>(cz) + 4 * cc + 2);
      const int nid[6] = {i0.x, i0.y, i0.z, i0.w, i1.x, i1.y};
      double x[6][3];
#pragma unroll
      for (int i = 0; i < 6; i++) ld_node(xc, nid[i], x[i]);
      double mp[3][3], R[3][3], aJ;
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int k = 0; k < 3; k++) mp[i][k] = mul(add(x[i][k], x[i + 3][k]), 0.5);
      cz_frame(mp[0], mp[1], mp[2], R, aJ);
#pragma unroll
      for (int n = 0; n < 3; n++)
#pragma unroll
        for (int k = 0; k < 3; k++) {
          const double xa = add(add(mul(x[n][0], R[k][0]), mul(x[n][1], R[k][1])), mul(x[n][2], R[k][2]));
          const double xb =
              add(add(mul(x[n + 3][0], R[k][0]), mul(x[n + 3][1], R[k][1])), mul(x[n + 3][2], R[k][2]));
          sD[t][3 * n + k] = sub(xa, xb);
        }
#pragma unroll
      for (int m = 0; m < 3; m++)
#pragma unroll
        for (int k = 0; k < 3; k++) sRJ[t][3 * m + k] = R[m][k];
      sRJ[t][9] = aJ;
    }
  }
  __syncthreads();
  const int j = t / 3, gp = t - 3 * j;
  const int c = blockIdx.x * CZ_PER_BLOCK + j;
  const bool live = c < nc && __ldg(czfail + c) == 0;
  double deln = P.deln, delt = P.delt, f_tn = P.f_tn, f_tt = P.f_tt;
  int fl = 0;
  if (live) {
    if (czprm) {
      const double4 w = czprm[c];
      f_tn = w.x; f_tt = w.y; deln = w.z; delt = w.w;
    }
    double pmax = __ldg(czs + 8 * (size_t)c + gp);
    double tmax = __ldg(czs + 8 * (size_t)c + 3 + gp);
    double R[3][3];
#pragma unroll
    for (int m = 0; m < 3; m++)
#pragma unroll
      for (int k = 0; k < 3; k++) R[m][k] = sRJ[j][3 * m + k];
    const double aJ = sRJ[j][9];
    // this Gauss point's opening
    double o[3] = {0, 0, 0};
#pragma unroll
    for (int n = 0; n < 3; n++) {
      const double sfn = P.sf[n * 3 + gp];
#pragma unroll
      for (int k = 0; k < 3; k++) o[k] = add(o[k], mul(sD[j][3 * n + k], sfn));
    }
    const double opn = o[2];
    const double opt = sqrt(add(mul(o[0], o[0]), mul(o[1], o[1])));
    // history axes from the cache (k_cz_hist), 6 doubles per Gauss point
    const double2 *hp = reinterpret_cast<const double2 *>(hist + 18 * (size_t)c + 6 * gp);
    const double2 h01 = __ldg(hp), h23 = __ldg(hp + 1), h45 = __ldg(hp + 2);
    const icf_axis Np{h01.x, h01.y, h23.x}, Tm{h23.y, h45.x, h45.y};
    bool undecided = false;
    const icf_law Lw = icf_cz_law_hist<EXACT>(LC, f_tn, f_tt, deln, delt, Np, Tm, pmax, tmax, opn, opt, undecided);
    // a failure comparison within rounding of its threshold: the library
    // repeats this assembly with the EXACT kernel (icf_read_counts)
    if (undecided) atomicAdd(counts + 5, 1);

    // local traction and its (symmetric) tangent (:301-340)
    double T[3], Td[3][3];
    if (opt < 1e-20) {
      T[0] = 0; T[1] = 0; T[2] = Lw.Tn;
      Td[0][0] = Lw.Dtt; Td[1][1] = Lw.Dtt; Td[2][2] = Lw.Dnn;
      Td[0][1] = Td[1][0] = 0;
      Td[0][2] = Td[2][0] = Lw.Dnt;
      Td[1][2] = Td[2][1] = Lw.Dnt;
    } else {
      const double io = 1.0 / opt;
      T[0] = Lw.Tt * o[0] * io;
      T[1] = Lw.Tt * o[1] * io;
      T[2] = Lw.Tn;
      const double io2 = io * io, io3 = io2 * io;
      const double u00 = o[0] * o[0], u10 = o[1] * o[0], u11 = o[1] * o[1];
      Td[0][0] = Lw.Dtt * u00 * io2 + Lw.Tt * u11 * io3;
      Td[1][1] = Lw.Dtt * u11 * io2 + Lw.Tt * u00 * io3;
      Td[2][2] = Lw.Dnn;
      Td[0][1] = Td[1][0] = Lw.Dtt * u10 * io2 - Lw.Tt * u10 * io3;
      Td[0][2] = Td[2][0] = Lw.Dnt * o[0] * io;
      Td[1][2] = Td[2][1] = Lw.Dnt * o[1] * io;
    }
    const double cw = (1.0 / 3.0) * aJ;
#pragma unroll
    for (int k = 0; k < 3; k++) sTw[t][k] = cw * (R[0][k] * T[0] + R[1][k] * T[1] + R[2][k] * T[2]);
    if (MIXED) {
      float Rf[3][3], TRf[3][3];
#pragma unroll
      for (int m = 0; m < 3; m++)
#pragma unroll
        for (int l = 0; l < 3; l++) Rf[m][l] = (float)R[m][l];
#pragma unroll
      for (int m = 0; m < 3; m++)
#pragma unroll
        for (int l = 0; l < 3; l++)
          TRf[m][l] = (float)Td[m][0] * Rf[0][l] + (float)Td[m][1] * Rf[1][l] + (float)Td[m][2] * Rf[2][l];
      const float cwf = (float)cw;
      int p = 0;
#pragma unroll
      for (int k = 0; k < 3; k++)
#pragma unroll
        for (int l = k; l < 3; l++)
          sQ[t][p++] = cwf * (Rf[0][k] * TRf[0][l] + Rf[1][k] * TRf[1][l] + Rf[2][k] * TRf[2][l]);
    } else {
      double TR[3][3];
#pragma unroll
      for (int m = 0; m < 3; m++)
#pragma unroll
        for (int l = 0; l < 3; l++) TR[m][l] = Td[m][0] * R[0][l] + Td[m][1] * R[1][l] + Td[m][2] * R[2][l];
      int p = 0;
#pragma unroll
      for (int k = 0; k < 3; k++)
#pragma unroll
        for (int l = k; l < 3; l++)
          sQ[t][p++] = cw * (R[0][k] * TR[0][l] + R[1][k] * TR[1][l] + R[2][k] * TR[2][l]);
    }
    sAv[t][0] = opn;
    sAv[t][1] = opt;
    sAv[t][2] = Lw.Tn;
    sAv[t][3] = Lw.Tt;
    sPT[t][0] = pmax;
    sPT[t][1] = tmax;
    const bool dmg = pmax >= deln * LC.rn || tmax >= delt * LC.rt;
    fl = (Lw.contact ? 1 : 0) | (Lw.failed ? 4 : 0) | (dmg ? 2 : 0);
  }
  sFl[t] = fl;
  __syncthreads();

  // combine the three Gauss points of CZ j: thread gp builds the Kt pairs
  // 2 gp and 2 gp + 1 (12 values), the rt row gp (3) and one pad value
  const int b3 = 3 * j;
  const bool failed = live && (((sFl[b3] | sFl[b3 + 1] | sFl[b3 + 2]) & 4) != 0);
  const bool on = live && !failed;
  double *so = sOut + j * ICF_CZ_STAGE;
#pragma unroll
  for (int hh = 0; hh < 2; hh++) {
    const int pr = 2 * gp + hh;
    const int pi = pr < 3 ? 0 : (pr < 5 ? 1 : 2);
    const int pj = pr < 3 ? pr : (pr < 5 ? pr - 2 : 2);
    double cf[3];
#pragma unroll
    for (int g = 0; g < 3; g++) cf[g] = P.sf[pi * 3 + g] * P.sf[pj * 3 + g];
#pragma unroll
    for (int comp = 0; comp < 6; comp++) {
      double val = 0.0;
      if (on) {
        if (MIXED) {
          float vf = 0.f;
#pragma unroll
          for (int g = 0; g < 3; g++) vf += (float)cf[g] * (float)sQ[b3 + g][comp];
          val = vf;
        } else {
#pragma unroll
          for (int g = 0; g < 3; g++) val += cf[g] * sQ[b3 + g][comp];
        }
      }
      so[6 * pr + comp] = val;
    }
  }
#pragma unroll
  for (int k = 0; k < 3; k++) {
    double val = 0.0;
    if (on)
#pragma unroll
      for (int g = 0; g < 3; g++) val += P.sf[gp * 3 + g] * sTw[b3 + g][k];
    so[36 + 3 * gp + k] = val;
  }
  so[45 + gp] = 0.0;
  int flag = 0;
  if (gp == 0 && live) {
    const int f0 = sFl[b3], f1 = sFl[b3 + 1], f2 = sFl[b3 + 2];
    const bool anyc = ((f0 | f1 | f2) & 1) != 0, damaged = ((f0 | f1 | f2) & 2) != 0;
    flag = (anyc ? 1 : 0) | ((!failed && damaged) ? 2 : 0) | (failed ? 4 : 0);
    czflags[c] = flag;
    cztent[2 * (size_t)c] = fmax(fmax(sPT[b3][0], sPT[b3 + 1][0]), sPT[b3 + 2][0]);
    cztent[2 * (size_t)c + 1] = fmax(fmax(sPT[b3][1], sPT[b3 + 1][1]), sPT[b3 + 2][1]);
    double av[4] = {0, 0, 0, 0};
    for (int g = 0; g < 3; g++)
      for (int k = 0; k < 4; k++) av[k] += sAv[b3 + g][k] / 3;
    reinterpret_cast<double4 *>(czavg)[c] =
        failed ? make_double4(0, 0, 0, 0) : make_double4(av[0], av[1], av[2], av[3]);
  } else if (gp == 0 && c < nc) {
    czflags[c] = 0;
  }
  __syncthreads();
  // coalesced store of the block's staging records
  const int c0 = blockIdx.x * CZ_PER_BLOCK;
  const int ncz = min(CZ_PER_BLOCK, nc - c0);
  if (!MIXED) {
    const int nvals = ncz * ICF_CZ_STAGE;
    double *dst = cs + (size_t)c0 * ICF_CZ_STAGE;
    for (int i = t; i < nvals; i += 3 * CZ_PER_BLOCK) dst[i] = sOut[i];
  } else {
    double *dr = cs + 12 * (size_t)c0;
    for (int i = t; i < 12 * ncz; i += 3 * CZ_PER_BLOCK) {
      const int jj = i / 12, q = i - 12 * jj;
      dr[i] = q < 9 ? sOut[jj * ICF_CZ_STAGE + 36 + q] : 0.0;
    }
    float *dk = reinterpret_cast<float *>(cs + 12 * (size_t)nc) + 36 * (size_t)c0;
    for (int i = t; i < 36 * ncz; i += 3 * CZ_PER_BLOCK) {
      const int jj = i / 36, q = i - 36 * jj;
      dk[i] = (float)sOut[jj * ICF_CZ_STAGE + q];
    }
  }
  // counters (integer atomics: order-independent)
  if (t < 32) {
    int dm = 0, fa = 0, ct = 0;
    for (int jj = t; jj < CZ_PER_BLOCK; jj += 32) {
      const int cc = c0 + jj;
      if (cc >= nc) continue;
      const int f0 = sFl[3 * jj], f1 = sFl[3 * jj + 1], f2 = sFl[3 * jj + 2];
      const int o = f0 | f1 | f2;
      const bool fl_ = (o & 4) != 0;
      dm += (!fl_ && (o & 2)) ? 1 : 0;
      fa += fl_ ? 1 : 0;
      ct += (o & 1) ? 1 : 0;
    }
    for (int d = 16; d > 0; d >>= 1) {
      dm += __shfl_down_sync(0xffffffffu, dm, d);
      fa += __shfl_down_sync(0xffffffffu, fa, d);
      ct += __shfl_down_sync(0xffffffffu, ct, d);
    }
    if (t == 0) {
      if (dm) atomicAdd(counts + 0, dm);
      if (fa) atomicAdd(counts + 1, fa);
      if (ct) atomicAdd(counts + 2, ct);
    }
  }
  (void)flag;
}

// A 72 B block or a 24 B rhs row (8 B aligned) in 16 B pieces: the split
// follows the address.
__device__ __forceinline__ void ld_blk9(const double *o, double b[9]) {
  if ((reinterpret_cast<uintptr_t>(o) & 8) == 0) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const double2 v = reinterpret_cast<const double2 *>(o)[k];
      b[2 * k] = v.x;
      b[2 * k + 1] = v.y;
    }
    b[8] = o[8];
  } else {
    b[0] = o[0];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const double2 v = reinterpret_cast<const double2 *>(o + 1)[k];
      b[1 + 2 * k] = v.x;
      b[2 + 2 * k] = v.y;
    }
  }
}
__device__ __forceinline__ void st_blk9(double *o, const double b[9]) {
  if ((reinterpret_cast<uintptr_t>(o) & 8) == 0) {
#pragma unroll
    for (int k = 0; k < 4; k++) reinterpret_cast<double2 *>(o)[k] = make_double2(b[2 * k], b[2 * k + 1]);
    o[8] = b[8];
  } else {
    o[0] = b[0];
#pragma unroll
    for (int k = 0; k < 4; k++) reinterpret_cast<double2 *>(o + 1)[k] = make_double2(b[1 + 2 * k], b[2 + 2 * k]);
  }
}
__device__ __forceinline__ void add_row3(double *o, const double v[3]) {
  if ((reinterpret_cast<uintptr_t>(o) & 8) == 0) {
    const double2 a = reinterpret_cast<const double2 *>(o)[0];
    reinterpret_cast<double2 *>(o)[0] = make_double2(a.x + v[0], a.y + v[1]);
    o[2] += v[2];
  } else {
    o[0] += v[0];
    const double2 a = reinterpret_cast<const double2 *>(o + 1)[0];
    reinterpret_cast<double2 *>(o + 1)[0] = make_double2(a.x + v[1], a.y + v[2]);
  }
}

// Impact contributions, one thread per block they touch: the records of the
// block's codes (k_imp_deriv writes them at the codes' positions in the
// slot-sorted list, so a block's records are contiguous; 96 B each, read as
// three 32 B loads; FP32-mixed: the FP32 block and the rhs in the first 64 B,
// two loads) are summed in FP64, in code order, and added to the block, and to
// the rhs row for a diagonal block (row >= 0).  A block that only contact
// pairs create (row == -2) is written, not added to: nothing else writes it.
// The touched blocks come in k_imp_add's order (icf_pattern.cu k_split_off):
// the launch over [first, first + count) reads its metadata contiguously.
__device__ __forceinline__ double4 ld_nc4(const double4 *p) {
  double4 r;
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(r.x), "=d"(r.y), "=d"(r.z), "=d"(r.w) : "l"(p));
  return r;
}
__device__ __forceinline__ double lo32(double w) { return (double)__int_as_float(__double2loint(w)); }
__device__ __forceinline__ double hi32(double w) { return (double)__int_as_float(__double2hiint(w)); }

template <bool MIXED>
__global__ void k_imp_add(int count, int first, const int2 *__restrict__ range, const int *__restrict__ pslot,
                          const int *__restrict__ row, const double *__restrict__ rec, double *__restrict__ vals,
                          double *__restrict__ rhs, int *__restrict__ nonfinite) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  bool bad = false;
  if (t < count) {
    const int w = first + t;
    const int2 qr = range[w];
    const int s = pslot[w], rw = row[w];
    double v[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int q = qr.x; q < qr.y; q++) {
      const double4 *R = reinterpret_cast<const double4 *>(rec + ICF_IMP_REC * (size_t)q);
      if (MIXED) {  // the block in FP32, two values per word, then the rhs
        const double4 a = ld_nc4(R), b = ld_nc4(R + 1);
        v[0] += lo32(a.x); v[1] += hi32(a.x); v[2] += lo32(a.y); v[3] += hi32(a.y);
        v[4] += lo32(a.z); v[5] += hi32(a.z); v[6] += lo32(a.w); v[7] += hi32(a.w);
        v[8] += lo32(b.x); v[9] += b.y; v[10] += b.z; v[11] += b.w;
      } else {
        double4 r[3];
#pragma unroll
        for (int k = 0; k < 3; k++) r[k] = ld_nc4(R + k);
#pragma unroll
        for (int k = 0; k < 3; k++) {
          v[4 * k] += r[k].x;
          v[4 * k + 1] += r[k].y;
          v[4 * k + 2] += r[k].z;
          v[4 * k + 3] += r[k].w;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < 9; k++) bad |= !isfinite(v[k]);
    double *o = vals + 9 * (size_t)s;
    if (rw == -2) {
      st_blk9(o, v);
    } else {
      double b[9];
      ld_blk9(o, b);
#pragma unroll
      for (int k = 0; k < 9; k++) b[k] += v[k];
      st_blk9(o, b);
    }
    if (rw >= 0) {
#pragma unroll
      for (int k = 0; k < 3; k++) bad |= !isfinite(v[9 + k]);
      add_row3(rhs + 3 * (size_t)rw, v + 9);
    }
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(nonfinite, 1);
}


// the impact add of the context's record format
using imp_add_fn = void (*)(int, int, const int2 *, const int *, const int *, const double *, double *, double *,
                            int *);
static imp_add_fn imp_add_for(const icf_ctx *ctx) {
  return ctx->precision == ICF_FP32_MIXED ? k_imp_add<true> : k_imp_add<false>;
}

// Node forces (the F field of the node array, GPU_Functionality.cs:519-527):
// per node the sum of the rhs of every tet vertex on it plus impact forces.
__global__ void k_node_force(int n, const int *__restrict__ off,
                             const int *__restrict__ inc,
                             const double4 *__restrict__ es,
                             const int *__restrict__ ioff,
                             const int *__restrict__ iinc,
                             const double *__restrict__ ks, int rstride, int roff,
                             double *__restrict__ F) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double f[3] = {0, 0, 0};
  for (int q = off[i]; q < off[i + 1]; q++) {
    const int code = inc[q];
    const double4 r = es[rstride * (size_t)(code >> 2) + roff + (code & 3)];
    f[0] += r.x;
    f[1] += r.y;
    f[2] += r.z;
  }
  if (ioff)
    for (int q = ioff[i]; q < ioff[i + 1]; q++) {
      const int code = iinc[q];
      const double *K = ks + (size_t)(code >> 2) * 12 + 3 * (code & 3);
      f[0] += K[0];
      f[1] += K[1];
      f[2] += K[2];
    }
  F[3 * (size_t)i + 0] = f[0];
  F[3 * (size_t)i + 1] = f[1];
  F[3 * (size_t)i + 2] = f[2];
}

// ---- node packing and Newmark kinematics ------------------------------------------
__global__ void k_pack_nodes(int n, const double4 *__restrict__ x0,
                             const double *__restrict__ un,
                             const double *__restrict__ vn,
                             const double *__restrict__ an,
                             double4 *__restrict__ xc, double2 *__restrict__ va) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 p = x0[i];
  xc[i] = make_double4(p.x + un[3 * i], p.y + un[3 * i + 1], p.z + un[3 * i + 2], 0.0);
  va[3 * i + 0] = make_double2(vn[3 * i], vn[3 * i + 1]);
  va[3 * i + 1] = make_double2(vn[3 * i + 2], an[3 * i]);
  va[3 * i + 2] = make_double2(an[3 * i + 1], an[3 * i + 2]);
}

// InferTentativeValues (Node.cs:79-97) fused with the node packing.
__global__ void k_infer(int n, double h, double beta, double gamma,
                        const double4 *__restrict__ x0,
                        const double *__restrict__ u, const double *__restrict__ v,
                        const double *__restrict__ a, const double *__restrict__ du,
                        double *__restrict__ un, double4 *__restrict__ xc,
                        double2 *__restrict__ va) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double unx[3], vnx[3], anx[3];
  for (int k = 0; k < 3; k++) {
    const size_t j = 3 * (size_t)i + k;
    unx[k] = u[j] + du[j];
    anx[k] = a[j] * (1.0 - 1.0 / (2 * beta)) + du[j] / (h * h * beta) + v[j] * (-1.0 / (h * beta));
    vnx[k] = v[j] + h * ((1.0 - gamma) * a[j] + gamma * anx[k]);
    un[j] = unx[k];
  }
  const double4 p = x0[i];
  xc[i] = make_double4(p.x + unx[0], p.y + unx[1], p.z + unx[2], 0.0);
  va[3 * i + 0] = make_double2(vnx[0], vnx[1]);
  va[3 * i + 1] = make_double2(vnx[2], anx[0]);
  va[3 * i + 2] = make_double2(anx[1], anx[2]);
}

__global__ void k_add_dx(int n, const int *__restrict__ alt,
                         const double *__restrict__ dx, double *__restrict__ du) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int r = alt[i];
  if (r < 0) return;
  for (int k = 0; k < 3; k++) du[3 * (size_t)i + k] += dx[3 * (size_t)r + k];
}

// sum of squares with a fixed reduction tree (deterministic)
__global__ void k_sumsq(int n, const double *__restrict__ x, double *__restrict__ part) {
  __shared__ double sh[256];
  double s = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    s += x[i] * x[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}
__global__ void k_sum_parts(int n, const double *__restrict__ part, double *out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0;
    for (int i = 0; i < n; i++) s += part[i];
    *out = s;
  }
}

// AcceptTentativeValues (Node.cs:62-77).
__global__ void k_accept(int n, double h, const double4 *__restrict__ x0,
                         double *__restrict__ u, double *__restrict__ v,
                         double *__restrict__ a, const double *__restrict__ un,
                         double *__restrict__ du, double4 *__restrict__ xc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double c[3];
  for (int k = 0; k < 3; k++) {
    const size_t j = 3 * (size_t)i + k;
    const double vnew = (un[j] - u[j]) / h;
    a[j] = (vnew - v[j]) / h;
    v[j] = vnew;
    u[j] = un[j];
    du[j] = 0;
    c[k] = u[j];
  }
  const double4 p = x0[i];
  xc[i] = make_double4(p.x + c[0], p.y + c[1], p.z + c[2], 0.0);
}

// Commit of the tentative CZ state (TransferUpdatedStateToHost, :496-516).
// History axes N(pmax/deln), T(tmax/delt) of every CZ Gauss point from the
// committed state: {Np.f, Np.d, Np.dd, Tm.f, Tm.d, Tm.dd} at hist[18c + 6gp].
__global__ void k_cz_hist(int nc, const double *__restrict__ czs, const double4 *__restrict__ czprm,
                          double deln0, double delt0, icf_law_c LC, double *__restrict__ hist) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * nc) return;
  const int c = t / 3, gp = t - 3 * c;
  double deln = deln0, delt = delt0;
  if (czprm) {
    const double4 w = czprm[c];
    deln = w.z;
    delt = w.w;
  }
  icf_axis Np, Tm;
  icf_cz_hist_axes(LC, deln, delt, czs[8 * (size_t)c + gp], czs[8 * (size_t)c + 3 + gp], Np, Tm);
  double *o = hist + 18 * (size_t)c + 6 * gp;
  o[0] = Np.f; o[1] = Np.d; o[2] = Np.dd;
  o[3] = Tm.f; o[4] = Tm.d; o[5] = Tm.dd;
}

__global__ void k_commit_cz(int nc, const double *__restrict__ tent,
                            const int *__restrict__ flags, double *__restrict__ czs,
                            int *__restrict__ fail) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc || fail[c]) return;
  if (flags[c] & 4) fail[c] = 1;
  for (int i = 0; i < 3; i++) {
    czs[8 * (size_t)c + i] = tent[2 * (size_t)c];
    czs[8 * (size_t)c + 3 + i] = tent[2 * (size_t)c + 1];
  }
}

// Non-failed committed CZs damaged at the level of _acceptFrame
// (ImplicitModel3.cs:304-317, CZ.damagedAtLevel, CZ.cs:13-16): pmax of the
// first Gauss point above deln lambda_n or tmax above delt lambda_t (per-CZ
// lengths with per-CZ strengths).
__global__ void k_count_damaged(int nc, const double *__restrict__ czs, const int *__restrict__ fail,
                                const double4 *__restrict__ czprm, double lambda_n, double lambda_t, double deln,
                                double delt, int *__restrict__ count) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc || fail[c]) return;
  const double dn = czprm ? czprm[c].z : deln, dt = czprm ? czprm[c].w : delt;
  if (czs[8 * (size_t)c] > dn * lambda_n || czs[8 * (size_t)c + 3] > dt * lambda_t) atomicAdd(count, 1);
}

}  // namespace

int icf_launch_count_damaged(icf_ctx *ctx, int *d_count) {
  ICF_CUDA(ctx, cudaMemsetAsync(d_count, 0, sizeof(int), ctx->stream));
  if (ctx->n_cz == 0) return ICF_OK;
  k_count_damaged<<<icf_blocks(ctx->n_cz, 256), 256, 0, ctx->stream>>>(
      ctx->n_cz, ctx->d_czs, ctx->d_czfail, ctx->per_cz_prm ? ctx->d_czprm : nullptr, ctx->prm.lambda_n,
      ctx->prm.lambda_t, ctx->prm.deln, ctx->prm.delt, d_count);
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}

namespace {
// Contribution layout (ICF_LAYOUT_CONTRIB): besides the compact rhs records
// es[4e + a] = {rhs_a, 0} (node forces), every tet writes each of its upper
// block contributions straight into the gather position tetpos[16e + 4a + b]:
//   off-diagonal (a != b): {h_a, V}, {h_b, 0}   FP64 64 B / FP32-mixed 32 B
//   diagonal (a == a):     {h_a, V}, {rhs_a, 0}  FP64 64 B / mixed 48 B
//                                                 ({h_a, V} FP32, rhs FP64)
// so the gathers read their inputs as contiguous streams.
template <int MINB, bool MIXED>
__global__ void __launch_bounds__(128, MINB)
    k_tet_contrib(int ne, const int4 *__restrict__ elem, const double4 *__restrict__ x0,
                  const double4 *__restrict__ xc, const double2 *__restrict__ va, icf_dprm P,
                  const int *__restrict__ tetpos, double4 *__restrict__ es, char *__restrict__ soff,
                  char *__restrict__ sdiag) {
  __shared__ double2 sbuf[4][32][17];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const long long base = (long long)blockIdx.x * blockDim.x + 32 * w;
  if (base >= ne) return;
  const int e = (int)base + lane;
  if (e < ne) {
    double2 *rec = sbuf[w][lane];
    tet_record<false>(e, elem, x0, xc, va, P, rec);
    const int4 *tp4 = reinterpret_cast<const int4 *>(tetpos + 16 * (size_t)e);
    int pos[16];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int4 t = __ldg(tp4 + q);
      pos[4 * q] = t.x; pos[4 * q + 1] = t.y; pos[4 * q + 2] = t.z; pos[4 * q + 3] = t.w;
    }
#pragma unroll
    for (int a = 0; a < 4; a++) {
      const double2 ha01 = rec[2 * a], ha2V = rec[2 * a + 1];
#pragma unroll
      for (int b = 0; b < 4; b++) {
        const int p = pos[4 * a + b];
        if (p < 0) continue;
        if (a == b) {
          const double2 r01 = rec[8 + 2 * a], r2 = rec[9 + 2 * a];
          if (MIXED) {
            char *d = sdiag + 48 * (size_t)p;
            *reinterpret_cast<float4 *>(d) = make_float4((float)ha01.x, (float)ha01.y, (float)ha2V.x, (float)ha2V.y);
            *reinterpret_cast<double2 *>(d + 16) = r01;
            *reinterpret_cast<double2 *>(d + 32) = r2;
          } else {
            double4 *d = reinterpret_cast<double4 *>(sdiag) + 2 * (size_t)p;
            d[0] = make_double4(ha01.x, ha01.y, ha2V.x, ha2V.y);
            d[1] = make_double4(r01.x, r01.y, r2.x, 0.0);
          }
        } else {
          const double2 hb01 = rec[2 * b], hb2V = rec[2 * b + 1];
          if (MIXED) {
            float4 *d = reinterpret_cast<float4 *>(soff) + 2 * (size_t)p;
            d[0] = make_float4((float)ha01.x, (float)ha01.y, (float)ha2V.x, (float)ha2V.y);
            d[1] = make_float4((float)hb01.x, (float)hb01.y, (float)hb2V.x, 0.f);
          } else {
            double4 *d = reinterpret_cast<double4 *>(soff) + 2 * (size_t)p;
            d[0] = make_double4(ha01.x, ha01.y, ha2V.x, ha2V.y);
            d[1] = make_double4(hb01.x, hb01.y, hb2V.x, 0.0);
          }
        }
      }
    }
  }
  __syncwarp();
  // compact rhs records, coalesced through shared memory
  const long long nrec = (ne - base) < 32 ? (ne - base) : 32;
  double2 *o = reinterpret_cast<double2 *>(es) + 8 * base;
#pragma unroll 4
  for (int k = 0; k < 8; k++) {
    const int idx = 32 * k + lane;
    if (idx < 8 * nrec) o[idx] = sbuf[w][idx >> 3][8 + (idx & 7)];
  }
}

struct tet_variant {
  const char *name;
  void (*fn)(int, const int4 *, const double4 *, const double4 *, const double2 *, icf_dprm, double4 *);
};
const tet_variant TET_VARIANTS[2][3] = {
    {{"t128 minb3", k_tet_unit<3, false>}, {"t128 minb2", k_tet_unit<2, false>}, {"t128 minb4", k_tet_unit<4, false>}},
    {{"t128 minb3", k_tet_unit<3, true>}, {"t128 minb2", k_tet_unit<2, true>}, {"t128 minb4", k_tet_unit<4, true>}},
};
typedef void (*tet_contrib_fn)(int, const int4 *, const double4 *, const double4 *, const double2 *, icf_dprm,
                               const int *, double4 *, char *, char *);
const tet_contrib_fn TET_CONTRIB[2][3] = {
    {k_tet_contrib<3, false>, k_tet_contrib<2, false>, k_tet_contrib<4, false>},
    {k_tet_contrib<3, true>, k_tet_contrib<2, true>, k_tet_contrib<4, true>},
};
constexpr int N_TET = 3;
}  // namespace

typedef void (*cz_fn)(int, const int *, const double4 *, const double *, const int *, const double4 *,
                      const double *, icf_dprm, icf_law_c, double *, double *, int *, double *, int *);
struct cz_variant {
  const char *name;
  cz_fn f64, f32;
};
const cz_variant CZ_VARIANTS[] = {
    {"96 thr minb1", k_cz_gp<false, 1>, k_cz_gp<true, 1>},
    {"96 thr minb6", k_cz_gp<false, 6>, k_cz_gp<true, 6>},
    {"96 thr minb8", k_cz_gp<false, 8>, k_cz_gp<true, 8>},
};
// the kernel that settles every failure comparison with the reference's
// rounding (the repeat of an assembly that left one undecided)
const cz_variant CZ_EXACT = {"96 thr exact", k_cz_gp<false, 1, true>, k_cz_gp<true, 1, true>};
constexpr int N_CZV = sizeof(CZ_VARIANTS) / sizeof(CZ_VARIANTS[0]);

int icf_tet_variants() { return N_TET; }
int icf_cz_variants() { return N_CZV; }
const char *icf_cz_variant_name(int v) { return CZ_VARIANTS[v].name; }

static icf_law_c make_law_c(const icf_ctx *ctx, const icf_dprm &P);

int icf_launch_cz(icf_ctx *ctx, int variant, const double4 *xc, double *cs, cudaStream_t s) {
  if (ctx->n_cz <= 0) return ICF_OK;
  if (variant < 0 || variant >= N_CZV) variant = 0;
  const icf_dprm P = icf_make_dprm(ctx);
  const icf_law_c LC = make_law_c(ctx, P);
  const cz_variant &V = ctx->cz_exact ? CZ_EXACT : CZ_VARIANTS[variant];
  const cz_fn f = ctx->precision == ICF_FP32_MIXED ? V.f32 : V.f64;
  f<<<icf_blocks(ctx->n_cz, CZ_PER_BLOCK), 3 * CZ_PER_BLOCK, 0, s>>>(
      ctx->n_cz, ctx->d_cz, xc, ctx->d_czs, ctx->d_czfail, ctx->per_cz_prm ? ctx->d_czprm : nullptr, ctx->d_czhist,
      P, LC, cs, ctx->d_cztent, ctx->d_czflags, ctx->d_czavg, ctx->d_counts);
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}
const char *icf_tet_variant_name(int v) { return TET_VARIANTS[0][v].name; }
int icf_launch_tet(icf_ctx *ctx, int variant, const double4 *xc, const double2 *va, double4 *es, cudaStream_t s) {
  if (ctx->n_elem <= 0) return ICF_OK;
  if (variant < 0 || variant >= N_TET) variant = 0;
  const icf_dprm P = icf_make_dprm(ctx);
  const int mixed = ctx->precision == ICF_FP32_MIXED ? 1 : 0;
  if (ctx->layout == ICF_LAYOUT_CONTRIB)
    TET_CONTRIB[mixed][variant]<<<icf_blocks(ctx->n_elem, 128), 128, 0, s>>>(
        ctx->n_elem, ctx->d_elem, ctx->d_x0, xc, va, P, ctx->d_tetpos, es,
        static_cast<char *>(ctx->d_stage_off), static_cast<char *>(ctx->d_stage_diag));
  else
    TET_VARIANTS[mixed][variant].fn<<<icf_blocks(ctx->n_elem, 128), 128, 0, s>>>(ctx->n_elem, ctx->d_elem,
                                                                                ctx->d_x0, xc, va, P, es);
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}

// ---- host launchers --------------------------------------------------------------
// One assembly as a fork/join DAG over three streams:
//   main : memsets | tets ............ | wait CZ -> diagonal gather | wait aux1 -> contact add
//          (diagonal and contact-only blocks) | join -> contact add (static off-diagonal blocks)
//   aux0 :         | CZs | wait tets -> off-diagonal gather ........|
//   aux1 :         | zero contact-only blocks, impact units .........|
// (or, per the tuner, both gathers on main, or one tiled gather, or split
// lists).  The unit kernels are occupancy- or latency-limited on their own, so
// running them side by side fills the machine; the gathers write disjoint
// blocks.
static icf_law_c make_law_c(const icf_ctx *ctx, const icf_dprm &P) {
  icf_law_c LC;
  LC.alpha = P.alpha; LC.beta = P.beta; LC.p_m = P.p_m; LC.p_n = P.p_n;
  LC.gam_n = P.gam_n; LC.gam_t = P.gam_t; LC.pMtn = P.pMtn; LC.pMnt = P.pMnt;
  LC.rn = P.rn; LC.rt = P.rt;
  const double *a0 = ctx->axis0;
  LC.N0 = icf_axis{a0[0], a0[1], a0[2], a0[3], a0[4], a0[5]};
  LC.T0 = icf_axis{a0[6], a0[7], a0[8], a0[9], a0[10], a0[11]};
  LC.zN = ctx->z0[0];
  LC.zT = ctx->z0[1];
  auto small_int = [](double v) { return (v == (double)(int)v && v >= 2 && v <= 16) ? (int)v : 0; };
  LC.alpha_int = small_int(P.alpha);
  LC.beta_int = small_int(P.beta);
  return LC;
}

// Refreshes the history-axis cache of the CZs when the damage state, the
// strengths or the constants changed since it was filled.
int icf_ensure_cz_hist(icf_ctx *ctx, cudaStream_t s) {
  if (ctx->hist_valid || ctx->n_cz == 0) return ICF_OK;
  const icf_dprm P = icf_make_dprm(ctx);
  k_cz_hist<<<icf_blocks(3LL * ctx->n_cz, 256), 256, 0, s>>>(ctx->n_cz, ctx->d_czs,
                                                           ctx->per_cz_prm ? ctx->d_czprm : nullptr, P.deln,
                                                           P.delt, make_law_c(ctx, P), ctx->d_czhist);
  ICF_CUDA(ctx, cudaGetLastError());
  ctx->hist_valid = true;
  return ICF_OK;
}

static int enqueue_assembly(icf_ctx *ctx, double h) {
  const icf_dprm P = icf_make_dprm(ctx);
  cudaStream_t s = ctx->stream, sa = ctx->aux[0], sb = ctx->aux[1];
  if (ctx->prof) sa = sb = s;  // per-kernel timing: one stream, in order
  cudaEvent_t e_fork = ctx->ev[0], e_cz = ctx->ev[1], e_tet = ctx->ev[2], e_a = ctx->ev[3],
              e_b = ctx->ev[4];
  ICF_CUDA(ctx, cudaMemsetAsync(ctx->d_counts, 0, 8 * sizeof(int), s));
  // the diagonal list gathers write every row's rhs (rows without a diagonal
  // block too); the row tiles hold only rows with one
  if (icf_tiles_active(ctx))
    ICF_CUDA(ctx, cudaMemsetAsync(ctx->d_rhs, 0, sizeof(double) * 3 * (size_t)ctx->N, s));
  if (ctx->prof) ICF_CUDA(ctx, cudaEventRecord(ctx->prof->ev[0], s));
  ICF_CUDA(ctx, cudaEventRecord(e_fork, s));
  ICF_CUDA(ctx, cudaStreamWaitEvent(sa, e_fork, 0));
  ICF_CUDA(ctx, cudaStreamWaitEvent(sb, e_fork, 0));

  // aux1: impact units
  if (ctx->n_imp > 0) {
    const int rc = icf_launch_imp_unit(ctx, sb);
    if (rc) return rc;
  }

  // main: tets (the fused row tiles compute them in place)
  const bool fused = icf_fused_active(ctx);
  if (ctx->n_elem > 0 && !fused)
    ICF_TRY_RC(icf_launch_tet(ctx, ctx->tune_tet, ctx->d_xc, ctx->d_va, ctx->d_es, s));
  // ids, node state (x0, x_t, v, a) once, 256 B record out
  const bool mixed = ctx->precision == ICF_FP32_MIXED;
  const bool contrib = ctx->layout == ICF_LAYOUT_CONTRIB;
  // per tet: the staging it writes (records, or rhs + contribution records)
  // and the part of it the off-diagonal and diagonal gathers read back
  long long tet_out, off_rec, diag_rec;
  if (contrib) {
    const long long ro = mixed ? 32 : 64, rd = mixed ? 48 : 64;
    tet_out = 64 * ctx->n_elem + 128 * ctx->n_elem + ro * 6 * ctx->n_elem + rd * 4 * ctx->n_elem;
    off_rec = ro * 6 * ctx->n_elem;
    diag_rec = rd * 4 * ctx->n_elem;
  } else {
    tet_out = (mixed ? 192 : 256) * ctx->n_elem;
    off_rec = (mixed ? 64 : 128) * ctx->n_elem;
    diag_rec = (mixed ? 192 : 256) * ctx->n_elem;
  }
  const long long cz_rec = mixed ? 240 : 8 * ICF_CZ_STAGE;
  if (ctx->n_elem > 0 && !fused)
    icf_prof_mark(ctx, s, "k_tet_unit", 16 * ctx->n_elem + tet_out + 112LL * ctx->n_nodes);
  ICF_CUDA(ctx, cudaEventRecord(e_tet, s));

  // aux0: CZs (on main ahead of the fused tiles, which need their staging)
  cudaStream_t scz = fused ? s : sa;
  if (ctx->n_cz > 0) {
    ICF_TRY_RC(icf_launch_cz(ctx, ctx->tune_cz, ctx->d_xc, ctx->d_cs, scz));
    // ids, six node positions, state in, per-CZ strengths, staging, tentative
    // state, flags and averages out
    icf_prof_mark(ctx, scz, "k_cz_gp", (24LL + 192 + 52 + (ctx->per_cz_prm ? 32 : 0) + cz_rec + 84) * ctx->n_cz);
  }
  ICF_CUDA(ctx, cudaEventRecord(e_cz, sa));

  const double nb = ctx->prm.NewmarkBeta, ng = ctx->prm.NewmarkGamma;
  const double sc = 1.0 + ctx->prm.dampingStiffness * ng / (h * nb);
  const double mc = (1.0 / (h * h) + ctx->prm.dampingMass * ng / h) / nb * (ctx->prm.rho / 20.0);
  // The gathers.  Algorithmic bytes of one list: its descriptors and blocks
  // (80 B per off-diagonal block, 104 B per row with its rhs), its codes, its
  // share (by codes) of the tet records and, for a list with CZ codes, the
  // CZ staging once.
  const icf_sell &OA = ctx->sell_off, &OB = ctx->sell_off_cz, &DA = ctx->sell_diag, &DB = ctx->sell_diag_cz;
  auto list_bytes = [&](const icf_sell &L, long long per_unit, long long rec, long long n_codes_all,
                        bool cz) {
    const double share = n_codes_all > 0 ? (double)L.n_real / (double)n_codes_all : 0.0;
    return per_unit * L.n_units + 4LL * L.n_real + (long long)(share * rec) + (cz ? cz_rec * ctx->n_cz : 0);
  };
  const long long codes_off = OA.n_real + OB.n_real, codes_diag = DA.n_real + DB.n_real;
  auto gather_off = [&](const icf_sell &L, cudaStream_t q, const char *name, bool cz) -> int {
    if (L.n_units == 0) return ICF_OK;
    ICF_TRY_RC(icf_launch_gather_off(ctx, L, ctx->tune_off, ctx->d_es, ctx->d_cs, sc, mc, P.lam, P.mu,
                                     ctx->d_vals, q));
    icf_prof_mark(ctx, q, name, list_bytes(L, 80, off_rec, codes_off, cz));
    return ICF_OK;
  };
  auto gather_diag = [&](const icf_sell &L, cudaStream_t q, const char *name, bool cz) -> int {
    if (L.n_units == 0) return ICF_OK;
    ICF_TRY_RC(icf_launch_gather_diag(ctx, L, ctx->tune_diag, ctx->d_es, ctx->d_cs, sc, mc, P.lam, P.mu,
                                      ctx->d_vals, ctx->d_rhs, q));
    icf_prof_mark(ctx, q, name, list_bytes(L, 104, diag_rec, codes_diag, cz));
    return ICF_OK;
  };
  if (fused) {
    // one kernel computes the tets of each row tile and writes every block;
    // algorithmic bytes: units, codes, the tets' ids and node state, the CZ
    // staging once
    const icf_tiles &T = ctx->tiles;
    ICF_TRY_RC(icf_launch_tile_fused(ctx, ctx->d_xc, ctx->d_va, ctx->d_cs, sc, mc, ctx->d_vals, ctx->d_rhs, s));
    icf_prof_mark(ctx, s, "k_tile_fused",
                  80 * T.n_off_units + 104 * T.n_diag_units + 4 * T.n_real + 16 * T.n_ttet + 112LL * ctx->n_nodes +
                      cz_rec * ctx->n_cz);
  } else if (icf_tiles_active(ctx)) {
    // one tiled gather for every block, once the tets and the CZs are staged;
    // algorithmic bytes: units, codes, the tet records and the CZ staging once
    const icf_tiles &T = ctx->tiles;
    ICF_CUDA(ctx, cudaStreamWaitEvent(s, e_cz, 0));
    ICF_TRY_RC(icf_launch_gather_tile(ctx, ctx->d_es, ctx->d_cs, sc, mc, P.lam, P.mu, ctx->d_vals, ctx->d_rhs, s));
    icf_prof_mark(ctx, s, "k_gather_tile",
                  80 * T.n_off_units + 104 * T.n_diag_units + 4 * T.n_real + diag_rec + cz_rec * ctx->n_cz);
  } else if (OB.n_units > 0 || DB.n_units > 0) {
    // split lists: the units without CZ codes run as soon as the tets are
    // staged, beside the CZ kernel (off-diagonal on aux1, diagonal on main);
    // the units with CZ codes wait for the CZs (off-diagonal on aux0,
    // diagonal on main)
    ICF_CUDA(ctx, cudaStreamWaitEvent(sb, e_tet, 0));
    ICF_TRY_RC(gather_off(OA, sb, "k_gather_off", false));
    ICF_TRY_RC(gather_diag(DA, s, "k_gather_diag", false));
    ICF_CUDA(ctx, cudaStreamWaitEvent(sa, e_tet, 0));
    ICF_TRY_RC(gather_off(OB, sa, "k_gather_off_cz", true));
    ICF_CUDA(ctx, cudaStreamWaitEvent(s, e_cz, 0));
    ICF_TRY_RC(gather_diag(DB, s, "k_gather_diag_cz", true));
  } else {
    // one list per gather: off-diagonal on aux0 once the tets are staged,
    // diagonal on main once the CZs are; or (serial_gathers) both on main,
    // one after the other
    cudaStream_t so = ctx->serial_gathers ? s : sa;
    if (ctx->serial_gathers) ICF_CUDA(ctx, cudaStreamWaitEvent(s, e_cz, 0));
    else ICF_CUDA(ctx, cudaStreamWaitEvent(sa, e_tet, 0));
    ICF_TRY_RC(gather_off(OA, so, "k_gather_off", true));
    ICF_CUDA(ctx, cudaStreamWaitEvent(s, e_cz, 0));
    ICF_TRY_RC(gather_diag(DA, s, "k_gather_diag", true));
  }
  ICF_CUDA(ctx, cudaEventRecord(e_a, sa));
  ICF_CUDA(ctx, cudaEventRecord(e_b, sb));
  // impact terms: the blocks that the off-diagonal gather does not write
  // (diagonal blocks, written on main, and contact-only blocks, zeroed on
  // aux1) as soon as the impacts are staged; the others after the join
  // algorithmic bytes: the impact staging once, 172 B per touched block and
  // 4 B per code, split between the two launches by their blocks
  const long long n_codes = 10LL * ctx->n_imp;  // at most; records of 12 doubles
  const long long imp_in = 8LL * ICF_IMP_REC * n_codes + 8LL * ctx->n_crs;
  const int n_a = ctx->n_crs - ctx->n_crs_off;
  ICF_CUDA(ctx, cudaStreamWaitEvent(s, e_b, 0));
  if (n_a > 0) {
    imp_add_for(ctx)<<<icf_blocks(n_a, 128), 128, 0, s>>>(n_a, 0, ctx->d_cr_range, ctx->d_cr_pslot, ctx->d_cr_row,
                                                  ctx->d_ks, ctx->d_vals, ctx->d_rhs, ctx->d_counts + 4);
    icf_prof_mark(ctx, s, "k_imp_add", imp_in * n_a / ctx->n_crs + 144LL * n_a);
  }
  ICF_CUDA(ctx, cudaStreamWaitEvent(s, e_a, 0));
  if (ctx->n_crs_off > 0 && ctx->n_crs > 0) {
    imp_add_for(ctx)<<<icf_blocks(ctx->n_crs_off, 128), 128, 0, s>>>(ctx->n_crs_off, n_a, ctx->d_cr_range,
                                                              ctx->d_cr_pslot, ctx->d_cr_row, ctx->d_ks,
                                                              ctx->d_vals, ctx->d_rhs, ctx->d_counts + 4);
    icf_prof_mark(ctx, s, "k_imp_add_off", imp_in * ctx->n_crs_off / ctx->n_crs + 144LL * ctx->n_crs_off);
  }

  ICF_CUDA(ctx, cudaGetLastError());
  ICF_CUDA(ctx, cudaMemcpyAsync(ctx->h_counts, ctx->d_counts, 8 * sizeof(int),
                                cudaMemcpyDeviceToHost, s));
  return ICF_OK;
}

// Launches the assembly, through the captured graph when enabled.  The graph
// is captured on first use and whenever the context's version (bumped by any
// call that changes the pattern, sizes, parameters or buffers) or the time
// step differs from the captured one.
void icf_prof_mark(icf_ctx *ctx, cudaStream_t s, const char *name, long long bytes) {
  icf_prof_state *p = ctx->prof;
  if (!p || p->n >= ICF_PROF_MAX) return;
  p->name[p->n] = name;
  p->bytes[p->n] = bytes;
  cudaEventRecord(p->ev[p->n + 1], s);
  p->n++;
}

// Runs `reps` assemblies without the graph, on one stream, with an event
// after every kernel; returns each kernel's mean device time.  The
// kernels, their launch shapes and their order are those of the graph; only
// the overlap between the streams is given up.
int icf_profile_assembly_impl(icf_ctx *ctx, double h, int reps, int *n, const char **names,
                              long long *bytes, double *ms) {
  icf_prof_state st;
  for (int i = 0; i <= ICF_PROF_MAX; i++) ICF_CUDA(ctx, cudaEventCreate(&st.ev[i]));
  std::vector<double> acc(ICF_PROF_MAX, 0.0);
  int rc = ICF_OK;
  rc = icf_ensure_cz_hist(ctx, ctx->stream);
  for (int r = 0; r < reps && rc == ICF_OK; r++) {
    st.n = 0;
    ctx->prof = &st;
    rc = enqueue_assembly(ctx, h);
    ctx->prof = nullptr;
    if (rc) break;
    const cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
      rc = icf_fail(ctx, ICF_ERR_CUDA, std::string("profile: ") + cudaGetErrorString(e));
      break;
    }
    for (int k = 0; k < st.n; k++) {
      float t = 0.f;
      cudaEventElapsedTime(&t, st.ev[k], st.ev[k + 1]);
      acc[k] += t;
    }
  }
  ctx->prof = nullptr;
  // the CZ history-axis refresh, which runs once per committed step (before
  // the next assembly), not once per assembly: timed on its own, reported last
  double hist_ms = 0.0;
  if (rc == ICF_OK && ctx->n_cz > 0 && st.n < ICF_PROF_MAX) {
    for (int r = 0; r < reps && rc == ICF_OK; r++) {
      ctx->hist_valid = false;
      cudaEventRecord(st.ev[0], ctx->stream);
      rc = icf_ensure_cz_hist(ctx, ctx->stream);
      cudaEventRecord(st.ev[1], ctx->stream);
      if (cudaEventSynchronize(st.ev[1]) != cudaSuccess) rc = icf_fail(ctx, ICF_ERR_CUDA, "profile: k_cz_hist");
      float t = 0.f;
      cudaEventElapsedTime(&t, st.ev[0], st.ev[1]);
      hist_ms += t;
    }
  }
  for (int i = 0; i <= ICF_PROF_MAX; i++) cudaEventDestroy(st.ev[i]);
  if (rc) return rc;
  *n = st.n;
  for (int k = 0; k < st.n; k++) {
    names[k] = st.name[k];
    bytes[k] = st.bytes[k];
    ms[k] = acc[k] / (reps > 0 ? reps : 1);
  }
  if (ctx->n_cz > 0 && st.n < ICF_PROF_MAX) {
    names[st.n] = "k_cz_hist";
    bytes[st.n] = 64LL * ctx->n_cz + 144LL * ctx->n_cz;  // committed state in, history axes out
    ms[st.n] = hist_ms / (reps > 0 ? reps : 1);
    *n = st.n + 1;
  }
  return ICF_OK;
}

int icf_launch_assembly(icf_ctx *ctx, double h) {
  ctx->last_h = h;
  ctx->n_law_exact = 0;
  ICF_TRY_RC(icf_ensure_cz_hist(ctx, ctx->stream));
  if (!ctx->use_graph) return enqueue_assembly(ctx, h);
  if (!ctx->graph_exec || ctx->graph_version != ctx->version || ctx->graph_h != h) {
    ICF_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue_assembly(ctx, h);
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(ctx->stream, &g);
    if (rc != ICF_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (ec != cudaSuccess) return icf_fail(ctx, ICF_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ec));
    // a new structure usually changes sizes and pointers only: update the
    // instantiated graph in place when its topology still matches, which
    // costs far less than instantiating anew
    if (ctx->graph_exec) {
      cudaGraphExecUpdateResultInfo info;
      if (cudaGraphExecUpdate(ctx->graph_exec, g, &info) == cudaSuccess) {
        cudaGraphDestroy(g);
        ctx->graph_version = ctx->version;
        ctx->graph_h = h;
        ICF_CUDA(ctx, cudaGraphLaunch(ctx->graph_exec, ctx->stream));
        return ICF_OK;
      }
      cudaGetLastError();  // the failed update leaves an error state behind
      cudaGraphExecDestroy(ctx->graph_exec);
      ctx->graph_exec = nullptr;
    }
    const cudaError_t ei = cudaGraphInstantiate(&ctx->graph_exec, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
      ctx->graph_exec = nullptr;
      return icf_fail(ctx, ICF_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
    }
    ctx->graph_version = ctx->version;
    ctx->graph_h = h;
  }
  ICF_CUDA(ctx, cudaGraphLaunch(ctx->graph_exec, ctx->stream));
  return ICF_OK;
}

int icf_launch_node_force(icf_ctx *ctx) {
  // the fused row tiles keep the tet rhs in shared memory: stage it for the
  // node sums (the node state is the last assembly's)
  if (icf_fused_active(ctx) && ctx->n_elem > 0)
    ICF_TRY_RC(icf_launch_tet(ctx, ctx->tune_tet, ctx->d_xc, ctx->d_va, ctx->d_es, ctx->stream));
  icf_node_inc t, m;
  int rc = icf_get_node_inc(ctx, &t, &m);
  if (rc) return rc;
  k_node_force<<<icf_blocks(ctx->n_nodes, 128), 128, 0, ctx->stream>>>(
      ctx->n_nodes, t.off, t.inc, ctx->d_es, ctx->n_imp > 0 ? m.off : nullptr, m.inc,
      ctx->n_imp > 0 ? icf_imp_forces(ctx->d_ks, ctx->n_imp) : nullptr,
      (ctx->precision == ICF_FP32_MIXED || ctx->layout == ICF_LAYOUT_CONTRIB) ? 4 : 8,
      (ctx->precision == ICF_FP32_MIXED || ctx->layout == ICF_LAYOUT_CONTRIB) ? 0 : 4, ctx->d_nodeF);
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}

int icf_launch_pack_nodes(icf_ctx *ctx, const double *d_un, const double *d_vn,
                          const double *d_an) {
  k_pack_nodes<<<icf_blocks(ctx->n_nodes, 256), 256, 0, ctx->stream>>>(
      ctx->n_nodes, ctx->d_x0, d_un, d_vn, d_an, ctx->d_xc, ctx->d_va);
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}

int icf_launch_infer(icf_ctx *ctx, double h) {
  k_infer<<<icf_blocks(ctx->n_nodes, 256), 256, 0, ctx->stream>>>(
      ctx->n_nodes, h, ctx->prm.NewmarkBeta, ctx->prm.NewmarkGamma, ctx->d_x0, ctx->d_u, ctx->d_v,
      ctx->d_a, ctx->d_du, ctx->d_un, ctx->d_xc, ctx->d_va);
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}

int icf_launch_add_dx(icf_ctx *ctx, const double *d_dx) {
  k_add_dx<<<icf_blocks(ctx->n_nodes, 256), 256, 0, ctx->stream>>>(ctx->n_nodes, ctx->d_alt, d_dx,
                                                                  ctx->d_du);
  const int n = 3 * ctx->N;
  const int nb = 256;
  k_sumsq<<<nb, 256, 0, ctx->stream>>>(n, d_dx, ctx->d_norm + 1);
  k_sum_parts<<<1, 32, 0, ctx->stream>>>(nb, ctx->d_norm + 1, ctx->d_norm);
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}

int icf_launch_sumsq(icf_ctx *ctx, const double *d_x, long long n) {
  k_sumsq<<<256, 256, 0, ctx->stream>>>((int)n, d_x, ctx->d_norm + 1);
  k_sum_parts<<<1, 32, 0, ctx->stream>>>(256, ctx->d_norm + 1, ctx->d_norm);
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}

int icf_launch_accept(icf_ctx *ctx, double h) {
  k_accept<<<icf_blocks(ctx->n_nodes, 256), 256, 0, ctx->stream>>>(
      ctx->n_nodes, h, ctx->d_x0, ctx->d_u, ctx->d_v, ctx->d_a, ctx->d_un, ctx->d_du, ctx->d_xc);
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}

int icf_launch_commit_cz(icf_ctx *ctx) {
  if (ctx->n_cz == 0) return ICF_OK;
  k_commit_cz<<<icf_blocks(ctx->n_cz, 256), 256, 0, ctx->stream>>>(
      ctx->n_cz, ctx->d_cztent, ctx->d_czflags, ctx->d_czs, ctx->d_czfail);
  ctx->hist_valid = false;
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}

// ---- launches with caller-chosen buffers (used by the allocation-free entry
// point in icf_noalloc.cu; the context's own assembly path above is separate)
static int enqueue_assembly_bufs(icf_ctx *ctx, double h, const icf_asm_bufs &B, cudaStream_t s);

// The caller-buffer path keeps the per-tet record layout (its scratch holds
// 256 B per tet; the contribution layout's staging lives in the context).
int icf_enqueue_assembly_bufs(icf_ctx *ctx, double h, const icf_asm_bufs &B, cudaStream_t s) {
  const int saved = ctx->layout;
  ctx->layout = ICF_LAYOUT_RECORDS;
  const int rc = enqueue_assembly_bufs(ctx, h, B, s);
  ctx->layout = saved;
  return rc;
}

static int enqueue_assembly_bufs(icf_ctx *ctx, double h, const icf_asm_bufs &B, cudaStream_t s) {
  ICF_TRY_RC(icf_ensure_cz_hist(ctx, s));
  const icf_dprm P = icf_make_dprm(ctx);
  ICF_CUDA(ctx, cudaMemsetAsync(ctx->d_counts, 0, 8 * sizeof(int), s));
  if (icf_tiles_active(ctx))
    ICF_CUDA(ctx, cudaMemsetAsync(B.rhs, 0, sizeof(double) * 3 * (size_t)ctx->N, s));
  k_pack_nodes<<<icf_blocks(ctx->n_nodes, 256), 256, 0, s>>>(ctx->n_nodes, ctx->d_x0, B.un, B.vn, B.an,
                                                            B.xc, B.va);
  const bool fused = icf_fused_active(ctx);
  if (ctx->n_elem > 0 && !fused)
    ICF_TRY_RC(icf_launch_tet(ctx, ctx->tune_tet, B.xc, B.va, B.es, s));
  if (ctx->n_cz > 0) {
    ICF_TRY_RC(icf_launch_cz(ctx, ctx->tune_cz, B.xc, B.cs, s));
  }
  if (ctx->n_imp > 0) {
    const int rc = icf_launch_imp_unit_bufs(ctx, B.xc, B.ks, s);
    if (rc) return rc;
  }
  const double nb = ctx->prm.NewmarkBeta, ng = ctx->prm.NewmarkGamma;
  const double sc = 1.0 + ctx->prm.dampingStiffness * ng / (h * nb);
  const double mc = (1.0 / (h * h) + ctx->prm.dampingMass * ng / h) / nb * (ctx->prm.rho / 20.0);
  if (fused) {
    ICF_TRY_RC(icf_launch_tile_fused(ctx, B.xc, B.va, B.cs, sc, mc, B.vals, B.rhs, s));
  } else if (icf_tiles_active(ctx)) {
    ICF_TRY_RC(icf_launch_gather_tile(ctx, B.es, B.cs, sc, mc, P.lam, P.mu, B.vals, B.rhs, s));
  } else {
    for (const icf_sell *L : {&ctx->sell_off, &ctx->sell_off_cz})
      if (L->n_units > 0)
        ICF_TRY_RC(icf_launch_gather_off(ctx, *L, ctx->tune_off, B.es, B.cs, sc, mc, P.lam, P.mu, B.vals, s));
    for (const icf_sell *L : {&ctx->sell_diag, &ctx->sell_diag_cz})
      if (L->n_units > 0)
        ICF_TRY_RC(icf_launch_gather_diag(ctx, *L, ctx->tune_diag, B.es, B.cs, sc, mc, P.lam, P.mu, B.vals,
                                          B.rhs, s));
  }
  if (ctx->n_crs > 0)
    imp_add_for(ctx)<<<icf_blocks(ctx->n_crs, 128), 128, 0, s>>>(ctx->n_crs, 0, ctx->d_cr_range, ctx->d_cr_pslot,
                                                        ctx->d_cr_row, B.ks, B.vals, B.rhs, ctx->d_counts + 4);

  ICF_CUDA(ctx, cudaGetLastError());
  ICF_CUDA(ctx, cudaMemcpyAsync(ctx->h_counts, ctx->d_counts, 8 * sizeof(int), cudaMemcpyDeviceToHost, s));
  return ICF_OK;
}

// ---- the cohesive law alone (icf_cz_law_eval) -------------------------------------
// One thread per Gauss-point state in[4i..4i+3] = {pmax, tmax, opn, opt}, with
// the history axes and the law exactly as k_cz_hist and k_cz_gp evaluate
// them: the fast law, and where it leaves a comparison undecided the exact
// one, as the repeated assembly would; out[7i..] = {pmax', tmax', Tn, Tt, Dnn,
// Dtt, Dnt}, fl[3i..] = {contact, failed, exact decision used}.
__global__ void k_cz_law_eval(int n, const double *__restrict__ in, const double4 *__restrict__ prm, icf_dprm P,
                              icf_law_c LC, double *__restrict__ out, int *__restrict__ fl) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double f_tn = P.f_tn, f_tt = P.f_tt, deln = P.deln, delt = P.delt;
  if (prm) {
    const double4 w = prm[i];
    f_tn = w.x; f_tt = w.y; deln = w.z; delt = w.w;
  }
  double pmax = in[4 * (size_t)i], tmax = in[4 * (size_t)i + 1];
  const double opn = in[4 * (size_t)i + 2], opt = in[4 * (size_t)i + 3];
  icf_axis Np, Tm;
  icf_cz_hist_axes(LC, deln, delt, pmax, tmax, Np, Tm);
  // the assembly reads the history axes back from the cache as {f, d, dd}
  const icf_axis Npc{Np.f, Np.d, Np.dd}, Tmc{Tm.f, Tm.d, Tm.dd};
  const double pmax0 = pmax, tmax0 = tmax;
  bool undecided = false;
  icf_law L = icf_cz_law_hist<false>(LC, f_tn, f_tt, deln, delt, Npc, Tmc, pmax, tmax, opn, opt, undecided);
  if (undecided) {
    pmax = pmax0;
    tmax = tmax0;
    bool u2 = false;
    L = icf_cz_law_hist<true>(LC, f_tn, f_tt, deln, delt, Npc, Tmc, pmax, tmax, opn, opt, u2);
  }
  double *o = out + 7 * (size_t)i;
  o[0] = pmax; o[1] = tmax; o[2] = L.Tn; o[3] = L.Tt; o[4] = L.Dnn; o[5] = L.Dtt; o[6] = L.Dnt;
  fl[3 * i] = L.contact ? 1 : 0;
  fl[3 * i + 1] = L.failed ? 1 : 0;
  fl[3 * i + 2] = undecided ? 1 : 0;
}

int icf_launch_law_eval(icf_ctx *ctx, int n, const double *in, const double4 *prm, double *out, int *fl) {
  const icf_dprm P = icf_make_dprm(ctx);
  k_cz_law_eval<<<icf_blocks(n, 128), 128, 0, ctx->stream>>>(n, in, prm, P, make_law_c(ctx, P), out, fl);
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}
