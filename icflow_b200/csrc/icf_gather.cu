// icf_gather.cu -- the atomic-free BCSR gathers and their launch variants.
//
// Each BCSR block (and rhs row) is written once by the lanes that own it,
// summing the contributions listed for it in the slot-sorted code lists of
// the pattern, laid out as sliced ELL (icf_sell).  This replaces the
// reference's per-entry CAS-loop atomics (AssembleBCSR12/18,
// element_kernels2.h:162-189, cz_kernels.h:177-203): the sum order is fixed,
// so the result is identical on every run.
//
// Every gather has several launch variants (registers per thread, codes per
// iteration, lanes per row).  They compute the same sums; the autotuner
// (icf_tune.cu) times them on the model at hand and keeps the fastest.
//
// Two precisions share the code.  FP64: staging records as k_tet_unit and
// k_cz_gp write them in FP64.  FP32-mixed: the Hessian inputs are FP32
// records (tet {h, V} as float4, CZ blocks Kt as float) and each block's tet
// and CZ terms are formed and summed in FP32, then written to the FP64 matrix;
// the rhs records and their sums stay FP64.
#include <cstdint>

#include "icf_internal.cuh"
#include "icf_tet.cuh"

namespace {

#ifndef CZ_UNROLL
#define CZ_UNROLL 2  // CZ codes per group in the gathers
#endif

__device__ __forceinline__ int sym_pair(int i, int j) {
  // (0,0)0 (0,1)1 (0,2)2 (1,1)3 (1,2)4 (2,2)5
  const int lo = i < j ? i : j, hi = i < j ? j : i;
  return lo == 0 ? hi : (lo == 1 ? 2 + hi : 5);
}

__device__ __forceinline__ void tet_code(uint32_t code, uint32_t &e, uint32_t &a, uint32_t &b) {
  e = (code >> 4) & 0x3FFFFFFu;
  a = (code >> 2) & 3u;
  b = code & 3u;
}

__device__ __forceinline__ void cz_code(uint32_t code, uint32_t &c, int &ia, int &ib, bool &same, bool &a_lo) {
  c = (code >> 6) & 0xFFFFFFu;
  const uint32_t a = (code >> 3) & 7u, bb = code & 7u;
  ia = a % 3;
  ib = bb % 3;
  same = (a < 3) == (bb < 3);
  a_lo = a < 3;
}

// One 32 B staging record in a single 256-bit read-only load (the record
// starts on a 32 B boundary: the staging buffer is 256 B aligned and every
// record is 32 B).
__device__ __forceinline__ double4 ld_rec(const double4 *p) {
  double4 v;
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(v.x), "=d"(v.y), "=d"(v.z), "=d"(v.w) : "l"(p));
  return v;
}

// Staging views and arithmetic of one precision.
struct fp64 {
  typedef double real;
  typedef double4 rec;
  const double4 *es;  // tet records: {h_a, V} at 8e + a, {rhs_a, 0} at 8e + 4 + a
  const double *cs;   // CZ records: Kt (6 x 6) at 48c, rt[3][3] at 48c + 36
  __device__ __forceinline__ rec hrec(uint32_t e, uint32_t a) const { return ld_rec(es + 8 * (size_t)e + a); }
  __device__ __forceinline__ const char *hsrc(uint32_t e) const {  // the 4 h records of tet e
    return reinterpret_cast<const char *>(es + 8 * (size_t)e);
  }
  __device__ __forceinline__ double4 rrec(uint32_t e, uint32_t a) const {
    return ld_rec(es + 8 * (size_t)e + 4 + a);
  }
  // Kt pair p sits at byte 384 c + 48 p: 32 B aligned for even p, 16 B past
  // a 32 B boundary for odd p, so two loads (32 B + 16 B) read its 48 B.
  __device__ __forceinline__ void kt(uint32_t c, int pair, real k[6]) const {
    const double *K = cs + (size_t)c * ICF_CZ_STAGE + 6 * pair;
    if ((pair & 1) == 0) {
      const double4 a = ld_rec(reinterpret_cast<const double4 *>(K));
      const double2 b = __ldg(reinterpret_cast<const double2 *>(K + 4));
      k[0] = a.x; k[1] = a.y; k[2] = a.z; k[3] = a.w; k[4] = b.x; k[5] = b.y;
    } else {
      const double2 a = __ldg(reinterpret_cast<const double2 *>(K));
      const double4 b = ld_rec(reinterpret_cast<const double4 *>(K + 2));
      k[0] = a.x; k[1] = a.y; k[2] = b.x; k[3] = b.y; k[4] = b.z; k[5] = b.w;
    }
  }
  __device__ __forceinline__ const double *rt(uint32_t c) const { return cs + (size_t)c * ICF_CZ_STAGE + 36; }
};
struct fp32mixed {
  typedef float real;
  typedef float4 rec;
  const float4 *es32;  // {h_a, V} at 4e + a
  const double4 *esr;  // {rhs_a, 0} at 4e + a
  const float *cs32;   // Kt at 36c
  const double *csr;   // rt at 12c
  __device__ __forceinline__ rec hrec(uint32_t e, uint32_t a) const { return es32[4 * (size_t)e + a]; }
  __device__ __forceinline__ const char *hsrc(uint32_t e) const {
    return reinterpret_cast<const char *>(es32 + 4 * (size_t)e);
  }
  __device__ __forceinline__ double4 rrec(uint32_t e, uint32_t a) const { return esr[4 * (size_t)e + a]; }
  __device__ __forceinline__ void kt(uint32_t c, int pair, real k[6]) const {
    const float2 *K2 = reinterpret_cast<const float2 *>(cs32 + (size_t)c * 36 + 6 * pair);
    const float2 k01 = __ldg(K2), k23 = __ldg(K2 + 1), k45 = __ldg(K2 + 2);
    k[0] = k01.x; k[1] = k01.y; k[2] = k23.x; k[3] = k23.y; k[4] = k45.x; k[5] = k45.y;
  }
  __device__ __forceinline__ const double *rt(uint32_t c) const { return csr + (size_t)c * 12; }
};

template <typename R>
struct gargs {
  R sc, mc, lam, mu;
};

// LHS_ab = stiffCoeff Df_ab + massCoeff M_ab rebuilt from the staging records
// {h_a, V} and {h_b, V} of one tet (k_tet_unit):
//   Df_ab = V (lam h_a h_b^T + mu h_b h_a^T + mu (h_a.h_b) I),
//   M_ab = rho/20 (1 + delta_ab) V I.
// A zero record (a padding code) adds nothing.
template <typename R, typename V4>
__device__ __forceinline__ void acc_tet(const V4 &A, const V4 &B, bool diag, const gargs<R> &g, R b[9]) {
  const R V = A.w;
  const R ha[3] = {A.x, A.y, A.z}, hb[3] = {B.x, B.y, B.z};
  const R dot = ha[0] * hb[0] + ha[1] * hb[1] + ha[2] * hb[2];
  const R c1 = g.sc * V * g.lam, c2 = g.sc * V * g.mu;
  const R cd = c2 * dot + g.mc * V * (diag ? R(2) : R(1));
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int l = 0; l < 3; l++) b[3 * k + l] += c1 * ha[k] * hb[l] + c2 * hb[k] * ha[l] + (k == l ? cd : R(0));
}

// Contribution of one CZ code: +-Kt[a mod 3][b mod 3] (symmetric 3x3) and,
// for a diagonal block, -+rt[a mod 3] (FP64).
template <typename S>
__device__ __forceinline__ void add_cz(const S &st, uint32_t code, typename S::real b[9], double *r) {
  typedef typename S::real R;
  uint32_t c;
  int ia, ib;
  bool same, a_lo;
  cz_code(code, c, ia, ib, same, a_lo);
  R k[6];
  st.kt(c, sym_pair(ia, ib), k);
  const R sg = same ? R(1) : R(-1);
  b[0] += sg * k[0]; b[1] += sg * k[1]; b[2] += sg * k[2];
  b[3] += sg * k[1]; b[4] += sg * k[3]; b[5] += sg * k[4];
  b[6] += sg * k[2]; b[7] += sg * k[4]; b[8] += sg * k[5];
  if (r != nullptr) {
    const double sa = a_lo ? -1.0 : 1.0;
    const double *rt = st.rt(c);
    r[0] += sa * __ldg(rt + 3 * ia + 0);
    r[1] += sa * __ldg(rt + 3 * ia + 1);
    r[2] += sa * __ldg(rt + 3 * ia + 2);
  }
}

// The CZ codes k0 .. k1 - 1 of a lane (stride 32), UC at a time: first the
// codes, then all their staging loads, then the terms in code order (the same
// terms and order as add_cz, code by code).
template <typename S, int UC>
__device__ __forceinline__ void cz_codes(const S &st, const uint32_t *c, int k0, int k1, typename S::real b[9],
                                         double *r) {
  typedef typename S::real R;
  for (int k = k0; k < k1; k += UC) {
    uint32_t cc[UC];
#pragma unroll
    for (int j = 0; j < UC; j++) cc[j] = (k + j < k1) ? __ldg(c + 32 * (k + j)) : ICF_CODE_PAD;
    R kk[UC][6], sg[UC];
    double rt[UC][3], sa[UC];
#pragma unroll
    for (int j = 0; j < UC; j++) {
      sg[j] = R(0);
      sa[j] = 0.0;
#pragma unroll
      for (int q = 0; q < 6; q++) kk[j][q] = R(0);
      rt[j][0] = rt[j][1] = rt[j][2] = 0.0;
      if (cc[j] != ICF_CODE_PAD) {
        uint32_t cz;
        int ia, ib;
        bool same, a_lo;
        cz_code(cc[j], cz, ia, ib, same, a_lo);
        st.kt(cz, sym_pair(ia, ib), kk[j]);
        sg[j] = same ? R(1) : R(-1);
        if (r != nullptr) {
          const double *p = st.rt(cz) + 3 * ia;
          rt[j][0] = __ldg(p);
          rt[j][1] = __ldg(p + 1);
          rt[j][2] = __ldg(p + 2);
          sa[j] = a_lo ? -1.0 : 1.0;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < UC; j++) {
      if (cc[j] == ICF_CODE_PAD) continue;
      const R g = sg[j];
      const R *K = kk[j];
      b[0] += g * K[0]; b[1] += g * K[1]; b[2] += g * K[2];
      b[3] += g * K[1]; b[4] += g * K[3]; b[5] += g * K[4];
      b[6] += g * K[2]; b[7] += g * K[4]; b[8] += g * K[5];
      if (r != nullptr) {
        r[0] += sa[j] * rt[j][0];
        r[1] += sa[j] * rt[j][1];
        r[2] += sa[j] * rt[j][2];
      }
    }
  }
}

// A 3x3 block (72 B, 8 B aligned) in five stores instead of nine: four
// 16 B stores from whichever of its first two doubles is 16 B aligned, and an
// rhs row (24 B) in two stores instead of three.
template <typename R>
__device__ __forceinline__ void st_block(double *__restrict__ vals, int s, const R b[9]) {
  double *o = vals + 9 * (size_t)s;
  if ((reinterpret_cast<uintptr_t>(o) & 8) == 0) {
    reinterpret_cast<double2 *>(o)[0] = make_double2((double)b[0], (double)b[1]);
    reinterpret_cast<double2 *>(o)[1] = make_double2((double)b[2], (double)b[3]);
    reinterpret_cast<double2 *>(o)[2] = make_double2((double)b[4], (double)b[5]);
    reinterpret_cast<double2 *>(o)[3] = make_double2((double)b[6], (double)b[7]);
    o[8] = (double)b[8];
  } else {
    o[0] = (double)b[0];
    reinterpret_cast<double2 *>(o + 1)[0] = make_double2((double)b[1], (double)b[2]);
    reinterpret_cast<double2 *>(o + 1)[1] = make_double2((double)b[3], (double)b[4]);
    reinterpret_cast<double2 *>(o + 1)[2] = make_double2((double)b[5], (double)b[6]);
    reinterpret_cast<double2 *>(o + 1)[3] = make_double2((double)b[7], (double)b[8]);
  }
}
__device__ __forceinline__ void st_rhs(double *__restrict__ rhs, int row, const double r[3]) {
  double *o = rhs + 3 * (size_t)row;
  if ((reinterpret_cast<uintptr_t>(o) & 8) == 0) {
    reinterpret_cast<double2 *>(o)[0] = make_double2(r[0], r[1]);
    o[2] = r[2];
  } else {
    o[0] = r[0];
    reinterpret_cast<double2 *>(o + 1)[0] = make_double2(r[1], r[2]);
  }
}

template <typename V4>
__device__ __forceinline__ V4 zero4();
template <>
__device__ __forceinline__ double4 zero4<double4>() { return make_double4(0, 0, 0, 0); }
template <>
__device__ __forceinline__ float4 zero4<float4>() { return make_float4(0, 0, 0, 0); }

// ---- off-diagonal blocks: one lane per block --------------------------------
// U codes per iteration; their 2U records are loaded before any is used.
template <typename S, int MINB, int U>
__global__ void __launch_bounds__(256, MINB)
    k_gather_off(int n_slices, const int4 *__restrict__ meta, const int2 *__restrict__ unit,
                 const uint32_t *__restrict__ codes, S st, gargs<typename S::real> g,
                 double *__restrict__ vals) {
  typedef typename S::real R;
  typedef typename S::rec V4;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= n_slices) return;
  const int4 m = meta[w];
  const uint32_t *c = codes + m.x + lane;
  R b[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int k = 0; k < m.y; k += U) {
    uint32_t cc[U];
#pragma unroll
    for (int j = 0; j < U; j++) cc[j] = (k + j < m.y) ? __ldg(c + 32 * (k + j)) : ICF_CODE_PAD;
    V4 A[U], B[U];
#pragma unroll
    for (int j = 0; j < U; j++) {
      A[j] = B[j] = zero4<V4>();
      if (cc[j] != ICF_CODE_PAD) {
        uint32_t e, a, bb;
        tet_code(cc[j], e, a, bb);
        A[j] = st.hrec(e, a);
        B[j] = st.hrec(e, bb);
      }
    }
#pragma unroll
    for (int j = 0; j < U; j++) acc_tet<R, V4>(A[j], B[j], false, g, b);
  }
  cz_codes<S, CZ_UNROLL>(st, c, m.y, m.y + m.z, b, nullptr);
  const int2 u = unit[32 * w + lane];
  if (u.x < 0) return;
  st_block(vals, u.x, b);
}

// ---- diagonal blocks and rhs rows: L lanes per row --------------------------
// Every code of a diagonal block has a == b: one {h, V} record for the block
// and one {rhs, 0} record for the row.  The L partial sums are combined by a
// fixed shuffle tree.
template <typename S, int L, int MINB, int U>
__global__ void __launch_bounds__(256, MINB)
    k_gather_diag(int n_slices, const int4 *__restrict__ meta, const int2 *__restrict__ unit,
                  const uint32_t *__restrict__ codes, S st, gargs<typename S::real> g,
                  double *__restrict__ vals, double *__restrict__ rhs, int *__restrict__ nonfinite) {
  typedef typename S::real R;
  typedef typename S::rec V4;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= n_slices) return;
  const int4 m = meta[w];
  const uint32_t *c = codes + m.x + lane;
  R b[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  double r[3] = {0, 0, 0};
  for (int k = 0; k < m.y; k += U) {
    uint32_t cc[U];
#pragma unroll
    for (int j = 0; j < U; j++) cc[j] = (k + j < m.y) ? __ldg(c + 32 * (k + j)) : ICF_CODE_PAD;
    V4 A[U];
    double4 Rr[U];
#pragma unroll
    for (int j = 0; j < U; j++) {
      A[j] = zero4<V4>();
      Rr[j] = make_double4(0, 0, 0, 0);
      if (cc[j] != ICF_CODE_PAD) {
        uint32_t e, a, bb;
        tet_code(cc[j], e, a, bb);
        A[j] = st.hrec(e, a);
        Rr[j] = st.rrec(e, a);
      }
    }
#pragma unroll
    for (int j = 0; j < U; j++) {
      acc_tet<R, V4>(A[j], A[j], true, g, b);
      r[0] += Rr[j].x;
      r[1] += Rr[j].y;
      r[2] += Rr[j].z;
    }
  }
  cz_codes<S, 1>(st, c, m.y, m.y + m.z, b, r);
#pragma unroll
  for (int o = 1; o < L; o <<= 1) {
#pragma unroll
    for (int q = 0; q < 9; q++) b[q] += __shfl_xor_sync(0xffffffffu, b[q], o);
#pragma unroll
    for (int q = 0; q < 3; q++) r[q] += __shfl_xor_sync(0xffffffffu, r[q], o);
  }
  const int sub = lane % L;
  const int2 u = unit[(32 / L) * w + lane / L];
  if (sub == 0 && u.x >= 0) {
    st_block(vals, u.x, b);
  }
  if (sub == (L > 1 ? 1 : 0) && u.y >= 0) {
    st_rhs(rhs, u.y, r);
  }
  // NaN/Inf check of the row (its rhs and diagonal block), one vote per warp
  bool bad = false;
  if (sub == 0)
#pragma unroll
    for (int q = 0; q < 9; q++) bad |= !isfinite((double)b[q]);
  bad |= !(isfinite(r[0]) && isfinite(r[1]) && isfinite(r[2]));
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(nonfinite, 1);
}

// ---- streaming cache hints ------------------------------------------------------
// Same as k_gather_off, but the list codes, units and the output blocks are
// touched once and go through L2 as evict-first (ld/st .cs), so that the
// staging records, which several blocks read, stay in L2 longer.
template <typename S, int MINB, int U>
__global__ void __launch_bounds__(256, MINB)
    k_gather_off_cs(int n_slices, const int4 *__restrict__ meta, const int2 *__restrict__ unit,
                    const uint32_t *__restrict__ codes, S st, gargs<typename S::real> g,
                    double *__restrict__ vals) {
  typedef typename S::real R;
  typedef typename S::rec V4;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= n_slices) return;
  const int4 m = __ldcs(meta + w);
  const uint32_t *c = codes + m.x + lane;
  R b[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int k = 0; k < m.y; k += U) {
    uint32_t cc[U];
#pragma unroll
    for (int j = 0; j < U; j++) cc[j] = (k + j < m.y) ? __ldcs(c + 32 * (k + j)) : ICF_CODE_PAD;
    V4 A[U], B[U];
#pragma unroll
    for (int j = 0; j < U; j++) {
      A[j] = B[j] = zero4<V4>();
      if (cc[j] != ICF_CODE_PAD) {
        uint32_t e, a, bb;
        tet_code(cc[j], e, a, bb);
        A[j] = st.hrec(e, a);
        B[j] = st.hrec(e, bb);
      }
    }
#pragma unroll
    for (int j = 0; j < U; j++) acc_tet<R, V4>(A[j], B[j], false, g, b);
  }
  for (int k = m.y; k < m.y + m.z; k++) {
    const uint32_t c0 = __ldcs(c + 32 * k);
    if (c0 != ICF_CODE_PAD) add_cz<S>(st, c0, b, nullptr);
  }
  const int2 u = __ldcs(unit + 32 * w + lane);
  if (u.x < 0) return;
  double *o = vals + 9 * (size_t)u.x;
#pragma unroll
  for (int q = 0; q < 9; q++) __stcs(o + q, (double)b[q]);
}

// ---- natural-order lists with coalesced block stores ---------------------------
// The slices hold 32 consecutive off-diagonal blocks, so their outputs are
// (nearly) contiguous in vals.  The lanes put their 9 values in shared memory
// and the warp stores the 288 values so that consecutive lanes write
// consecutive doubles: a few L2 write requests per warp instead of one per
// sector.  The price is divergence: a slice runs as many iterations as its
// longest list.
template <typename S, int MINB, int U>
__global__ void __launch_bounds__(256, MINB)
    k_gather_off_nat(int n_slices, const int4 *__restrict__ meta, const int2 *__restrict__ unit,
                     const uint32_t *__restrict__ codes, S st, gargs<typename S::real> g,
                     double *__restrict__ vals) {
  typedef typename S::real R;
  typedef typename S::rec V4;
  __shared__ double sb[8][32 * 9];
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= n_slices) return;
  const int wl = threadIdx.x >> 5;
  const int4 m = meta[w];
  const int2 u = unit[32 * w + lane];
  const uint32_t *c = codes + m.x + lane;
  R b[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int k = 0; k < m.y; k += U) {
    uint32_t cc[U];
#pragma unroll
    for (int j = 0; j < U; j++) cc[j] = (k + j < m.y) ? __ldg(c + 32 * (k + j)) : ICF_CODE_PAD;
    V4 A[U], B[U];
#pragma unroll
    for (int j = 0; j < U; j++) {
      A[j] = B[j] = zero4<V4>();
      if (cc[j] != ICF_CODE_PAD) {
        uint32_t e, a, bb;
        tet_code(cc[j], e, a, bb);
        A[j] = st.hrec(e, a);
        B[j] = st.hrec(e, bb);
      }
    }
#pragma unroll
    for (int j = 0; j < U; j++) acc_tet<R, V4>(A[j], B[j], false, g, b);
  }
  cz_codes<S, CZ_UNROLL>(st, c, m.y, m.y + m.z, b, nullptr);
#pragma unroll
  for (int q = 0; q < 9; q++) sb[wl][9 * lane + q] = (double)b[q];
  __syncwarp();
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const int idx = 32 * k + lane;
    const int blk = idx / 9, q = idx - 9 * blk;
    const int slot = __shfl_sync(0xffffffffu, u.x, blk);
    if (slot >= 0) vals[9 * (size_t)slot + q] = sb[wl][idx];
  }
}

// ---- persistent, software-pipelined variants --------------------------------
// A warp walks slices w, w + W, ... (W = warps in the grid).  While the
// records of slice w are in flight it already loads the next slice's meta,
// unit and first codes, so the dependent chain meta -> codes -> records is
// paid about once per slice instead of three times.
template <typename S, int MINB, int U>
__global__ void __launch_bounds__(256, MINB)
    k_gather_off_pipe(int n_slices, const int4 *__restrict__ meta, const int2 *__restrict__ unit,
                      const uint32_t *__restrict__ codes, S st, gargs<typename S::real> g,
                      double *__restrict__ vals) {
  typedef typename S::real R;
  typedef typename S::rec V4;
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= n_slices) return;
  int4 m = meta[w];
  int2 u = unit[32 * w + lane];
  uint32_t cc[U];
#pragma unroll
  for (int j = 0; j < U; j++) cc[j] = j < m.y ? __ldg(codes + m.x + 32 * j + lane) : ICF_CODE_PAD;
  while (true) {
    const int wn = w + nw;
    int4 mn = make_int4(0, 0, 0, 0);
    int2 un = make_int2(-1, -1);
    if (wn < n_slices) {
      mn = meta[wn];
      un = unit[32 * wn + lane];
    }
    V4 A[U], B[U];
#pragma unroll
    for (int j = 0; j < U; j++) {
      A[j] = B[j] = zero4<V4>();
      if (cc[j] != ICF_CODE_PAD) {
        uint32_t e, a, bb;
        tet_code(cc[j], e, a, bb);
        A[j] = st.hrec(e, a);
        B[j] = st.hrec(e, bb);
      }
    }
    uint32_t cn[U];
#pragma unroll
    for (int j = 0; j < U; j++) cn[j] = (wn < n_slices && j < mn.y) ? __ldg(codes + mn.x + 32 * j + lane) : ICF_CODE_PAD;
    R b[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int j = 0; j < U; j++) acc_tet<R, V4>(A[j], B[j], false, g, b);
    const uint32_t *c = codes + m.x + lane;
    for (int k = U; k < m.y; k++) {
      const uint32_t c0 = __ldg(c + 32 * k);
      if (c0 != ICF_CODE_PAD) {
        uint32_t e, a, bb;
        tet_code(c0, e, a, bb);
        acc_tet<R, V4>(st.hrec(e, a), st.hrec(e, bb), false, g, b);
      }
    }
    cz_codes<S, CZ_UNROLL>(st, c, m.y, m.y + m.z, b, nullptr);
    if (u.x >= 0) {
      st_block(vals, u.x, b);
    }
    if (wn >= n_slices) break;
    w = wn;
    m = mn;
    u = un;
#pragma unroll
    for (int j = 0; j < U; j++) cc[j] = cn[j];
  }
}

template <typename S, int L, int MINB, int U>
__global__ void __launch_bounds__(256, MINB)
    k_gather_diag_pipe(int n_slices, const int4 *__restrict__ meta, const int2 *__restrict__ unit,
                       const uint32_t *__restrict__ codes, S st, gargs<typename S::real> g,
                       double *__restrict__ vals, double *__restrict__ rhs, int *__restrict__ nonfinite) {
  typedef typename S::real R;
  typedef typename S::rec V4;
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= n_slices) return;
  int4 m = meta[w];
  int2 u = unit[(32 / L) * w + lane / L];
  uint32_t cc[U];
#pragma unroll
  for (int j = 0; j < U; j++) cc[j] = j < m.y ? __ldg(codes + m.x + 32 * j + lane) : ICF_CODE_PAD;
  bool bad = false;
  while (true) {
    const int wn = w + nw;
    int4 mn = make_int4(0, 0, 0, 0);
    int2 un = make_int2(-1, -1);
    if (wn < n_slices) {
      mn = meta[wn];
      un = unit[(32 / L) * wn + lane / L];
    }
    V4 A[U];
    double4 Rr[U];
#pragma unroll
    for (int j = 0; j < U; j++) {
      A[j] = zero4<V4>();
      Rr[j] = make_double4(0, 0, 0, 0);
      if (cc[j] != ICF_CODE_PAD) {
        uint32_t e, a, bb;
        tet_code(cc[j], e, a, bb);
        A[j] = st.hrec(e, a);
        Rr[j] = st.rrec(e, a);
      }
    }
    uint32_t cn[U];
#pragma unroll
    for (int j = 0; j < U; j++) cn[j] = (wn < n_slices && j < mn.y) ? __ldg(codes + mn.x + 32 * j + lane) : ICF_CODE_PAD;
    R b[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double r[3] = {0, 0, 0};
#pragma unroll
    for (int j = 0; j < U; j++) {
      acc_tet<R, V4>(A[j], A[j], true, g, b);
      r[0] += Rr[j].x;
      r[1] += Rr[j].y;
      r[2] += Rr[j].z;
    }
    const uint32_t *c = codes + m.x + lane;
    for (int k = U; k < m.y; k++) {
      const uint32_t c0 = __ldg(c + 32 * k);
      if (c0 != ICF_CODE_PAD) {
        uint32_t e, a, bb;
        tet_code(c0, e, a, bb);
        const V4 A1 = st.hrec(e, a);
        const double4 R1 = st.rrec(e, a);
        acc_tet<R, V4>(A1, A1, true, g, b);
        r[0] += R1.x;
        r[1] += R1.y;
        r[2] += R1.z;
      }
    }
    cz_codes<S, 1>(st, c, m.y, m.y + m.z, b, r);
#pragma unroll
    for (int o = 1; o < L; o <<= 1) {
#pragma unroll
      for (int q = 0; q < 9; q++) b[q] += __shfl_xor_sync(0xffffffffu, b[q], o);
#pragma unroll
      for (int q = 0; q < 3; q++) r[q] += __shfl_xor_sync(0xffffffffu, r[q], o);
    }
    const int sub = lane % L;
    if (sub == 0 && u.x >= 0) {
      st_block(vals, u.x, b);
    }
    if (sub == (L > 1 ? 1 : 0) && u.y >= 0) {
      st_rhs(rhs, u.y, r);
    }
    if (sub == 0)
#pragma unroll
      for (int q = 0; q < 9; q++) bad |= !isfinite((double)b[q]);
    bad |= !(isfinite(r[0]) && isfinite(r[1]) && isfinite(r[2]));
    if (wn >= n_slices) break;
    w = wn;
    m = mn;
    u = un;
#pragma unroll
    for (int j = 0; j < U; j++) cc[j] = cn[j];
  }
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(nonfinite, 1);
}

// ---- contribution layout (ICF_LAYOUT_CONTRIB) --------------------------------
// The tet kernel wrote each contribution's inputs at its list position, so
// iteration k of lane l reads record (meta.x + 32 k + l): one contiguous
// stream per warp, no codes and no random loads for the tet part.
// Positions of padding codes hold zero records.
template <bool MIXED>
struct crec;
template <>
struct crec<false> {
  typedef double4 V4;
  static __device__ __forceinline__ void off(const char *st, long long p, V4 &A, V4 &B) {
    const double4 *r = reinterpret_cast<const double4 *>(st) + 2 * p;
    A = r[0];
    B = r[1];
  }
  static __device__ __forceinline__ void diag(const char *st, long long p, V4 &A, double4 &R) {
    const double4 *r = reinterpret_cast<const double4 *>(st) + 2 * p;
    A = r[0];
    R = r[1];
  }
};
template <>
struct crec<true> {
  typedef float4 V4;
  static __device__ __forceinline__ void off(const char *st, long long p, V4 &A, V4 &B) {
    const float4 *r = reinterpret_cast<const float4 *>(st) + 2 * p;
    A = r[0];
    B = r[1];
  }
  static __device__ __forceinline__ void diag(const char *st, long long p, V4 &A, double4 &R) {
    const char *r = st + 48 * p;
    A = *reinterpret_cast<const float4 *>(r);
    const double2 r01 = *reinterpret_cast<const double2 *>(r + 16);
    const double2 r2 = *reinterpret_cast<const double2 *>(r + 32);
    R = make_double4(r01.x, r01.y, r2.x, 0.0);
  }
};

template <typename S, bool MIXED, int MINB, int U>
__global__ void __launch_bounds__(256, MINB)
    k_gather_off_c(int n_slices, const int4 *__restrict__ meta, const int2 *__restrict__ unit,
                   const uint32_t *__restrict__ codes, const char *__restrict__ stage, S st,
                   gargs<typename S::real> g, double *__restrict__ vals) {
  typedef typename S::real R;
  typedef typename crec<MIXED>::V4 V4;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= n_slices) return;
  const int4 m = meta[w];
  R b[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const long long p0 = (long long)m.x + lane;
  for (int k = 0; k < m.y; k += U) {
    V4 A[U], B[U];
#pragma unroll
    for (int j = 0; j < U; j++) {
      A[j] = B[j] = zero4<V4>();
      if (k + j < m.y) crec<MIXED>::off(stage, p0 + 32LL * (k + j), A[j], B[j]);
    }
#pragma unroll
    for (int j = 0; j < U; j++) acc_tet<R, V4>(A[j], B[j], false, g, b);
  }
  const uint32_t *c = codes + m.x + lane;
  cz_codes<S, CZ_UNROLL>(st, c, m.y, m.y + m.z, b, nullptr);
  const int2 u = unit[32 * w + lane];
  if (u.x < 0) return;
  st_block(vals, u.x, b);
}

template <typename S, bool MIXED, int L, int MINB, int U>
__global__ void __launch_bounds__(256, MINB)
    k_gather_diag_c(int n_slices, const int4 *__restrict__ meta, const int2 *__restrict__ unit,
                    const uint32_t *__restrict__ codes, const char *__restrict__ stage, S st,
                    gargs<typename S::real> g, double *__restrict__ vals, double *__restrict__ rhs,
                    int *__restrict__ nonfinite) {
  typedef typename S::real R;
  typedef typename crec<MIXED>::V4 V4;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= n_slices) return;
  const int4 m = meta[w];
  R b[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  double r[3] = {0, 0, 0};
  const long long p0 = (long long)m.x + lane;
  for (int k = 0; k < m.y; k += U) {
    V4 A[U];
    double4 Rr[U];
#pragma unroll
    for (int j = 0; j < U; j++) {
      A[j] = zero4<V4>();
      Rr[j] = make_double4(0, 0, 0, 0);
      if (k + j < m.y) crec<MIXED>::diag(stage, p0 + 32LL * (k + j), A[j], Rr[j]);
    }
#pragma unroll
    for (int j = 0; j < U; j++) {
      acc_tet<R, V4>(A[j], A[j], true, g, b);
      r[0] += Rr[j].x;
      r[1] += Rr[j].y;
      r[2] += Rr[j].z;
    }
  }
  const uint32_t *c = codes + m.x + lane;
  cz_codes<S, 1>(st, c, m.y, m.y + m.z, b, r);
#pragma unroll
  for (int o = 1; o < L; o <<= 1) {
#pragma unroll
    for (int q = 0; q < 9; q++) b[q] += __shfl_xor_sync(0xffffffffu, b[q], o);
#pragma unroll
    for (int q = 0; q < 3; q++) r[q] += __shfl_xor_sync(0xffffffffu, r[q], o);
  }
  const int sub = lane % L;
  const int2 u = unit[(32 / L) * w + lane / L];
  if (sub == 0 && u.x >= 0) {
    st_block(vals, u.x, b);
  }
  if (sub == (L > 1 ? 1 : 0) && u.y >= 0) {
    st_rhs(rhs, u.y, r);
  }
  // NaN/Inf check of the row (its rhs and diagonal block), one vote per warp
  bool bad = false;
  if (sub == 0)
#pragma unroll
    for (int q = 0; q < 9; q++) bad |= !isfinite((double)b[q]);
  bad |= !(isfinite(r[0]) && isfinite(r[1]) && isfinite(r[2]));
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(nonfinite, 1);
}

// ---- variant tables ---------------------------------------------------------
template <typename S>
using off_fn = void (*)(int, const int4 *, const int2 *, const uint32_t *, S, gargs<typename S::real>, double *);
template <typename S>
using diag_fn = void (*)(int, const int4 *, const int2 *, const uint32_t *, S, gargs<typename S::real>, double *,
                         double *, int *);

template <typename S>
using offc_fn = void (*)(int, const int4 *, const int2 *, const uint32_t *, const char *, S,
                         gargs<typename S::real>, double *);
template <typename S>
using diagc_fn = void (*)(int, const int4 *, const int2 *, const uint32_t *, const char *, S,
                          gargs<typename S::real>, double *, double *, int *);

struct off_variant {
  const char *name;
  off_fn<fp64> f64;
  off_fn<fp32mixed> f32;
  offc_fn<fp64> c64;
  offc_fn<fp32mixed> c32;
  int persistent_minb;  // > 0: persistent grid of n_sm * this many blocks (record layout)
  bool natural;         // reads natural-order lists
};
struct diag_variant {
  const char *name;
  int lanes;
  diag_fn<fp64> f64;
  diag_fn<fp32mixed> f32;
  diagc_fn<fp64> c64;
  diagc_fn<fp32mixed> c32;
  int persistent_minb;
};

// ---- row tiles (icf_tiles): every block of a set of rows per CTA ---------------
__device__ __forceinline__ void cp16(void *smem, const void *gmem) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// The CTA first copies, with asynchronous 16 B copies, the tile's slice
// metadata, units and 16-bit tet codes (contiguous ranges) and the {h_a, V}
// records of its tets (one 128 B / 64 B line per tet) into shared memory.
// Its warps then take the tile's slices in turn, one lane per block.  A tet
// code names the tet's position in the tile; CZ codes are read from global
// memory.  Diagonal blocks (unit row >= 0) also sum their vertices' rhs
// records and the CZ rt terms.  Per block, the sum runs over the codes in the
// order of the static code list, as in the list gathers.
#define TILE_THREADS 256
template <typename S, int MINB, int U>
__global__ void __launch_bounds__(TILE_THREADS, MINB)
    k_gather_tile(const int4 *__restrict__ tiles, const int2 *__restrict__ trange, const int *__restrict__ ttet,
                  const int4 *__restrict__ meta, const int2 *__restrict__ unit, const uint16_t *__restrict__ tcodes,
                  const uint32_t *__restrict__ czcodes, S st, gargs<typename S::real> g,
                  double *__restrict__ vals, double *__restrict__ rhs, int *__restrict__ nonfinite) {
  typedef typename S::real R;
  typedef typename S::rec V4;
  constexpr int CH = 4 * (int)sizeof(V4) / 16;  // 16 B chunks per tet
  extern __shared__ __align__(16) unsigned char tile_smem[];
  __shared__ int next_slice;
  const int4 t = tiles[blockIdx.x];
  const int2 tr = trange[blockIdx.x];
  V4 *sh = reinterpret_cast<V4 *>(tile_smem);
  int4 *smeta = reinterpret_cast<int4 *>(sh + 4 * t.y);
  int2 *sunit = reinterpret_cast<int2 *>(smeta + t.w);
  uint16_t *scode = reinterpret_cast<uint16_t *>(sunit + 32 * t.w);
  int *gid = reinterpret_cast<int *>(scode + tr.y);
  const int tid = threadIdx.x, nth = blockDim.x;
  for (int q = tid; q < t.w; q += nth) cp16(smeta + q, meta + t.z + q);
  for (int q = tid; q < 16 * t.w; q += nth) cp16(sunit + 2 * q, unit + 32 * (size_t)t.z + 2 * q);
  for (int q = tid; q < tr.y / 8; q += nth) cp16(scode + 8 * q, tcodes + tr.x + 8 * q);
  {
    // thread tid copies chunk tid % CH of tets tid / CH, tid / CH + nth / CH, ...
    const int ch = tid % CH, step = nth / CH;
    int k = tid / CH;
    for (; k + 3 * step < t.y; k += 4 * step) {
      int e[4];
#pragma unroll
      for (int j = 0; j < 4; j++) e[j] = __ldg(ttet + t.x + k + j * step);
#pragma unroll
      for (int j = 0; j < 4; j++) {
        cp16(reinterpret_cast<char *>(sh + 4 * (k + j * step)) + 16 * ch, st.hsrc((uint32_t)e[j]) + 16 * ch);
        if (ch == 0) gid[k + j * step] = e[j];
      }
    }
    for (; k < t.y; k += step) {
      const int e = __ldg(ttet + t.x + k);
      cp16(reinterpret_cast<char *>(sh + 4 * k) + 16 * ch, st.hsrc((uint32_t)e) + 16 * ch);
      if (ch == 0) gid[k] = e;
    }
  }
  if (tid == 0) next_slice = nth >> 5;
  cp_wait_all();
  __syncthreads();
  const int lane = tid & 31;
  bool bad = false;
  int w = tid >> 5;
  while (w < t.w) {
    const int4 m = smeta[w];
    const int2 u = sunit[32 * w + lane];
    const bool dg = u.y >= 0;
    const uint16_t *c = scode + (m.x - tr.x) + lane;
    R b[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double r[3] = {0, 0, 0};
    for (int k = 0; k < m.y; k += U) {
      uint32_t cc[U];
#pragma unroll
      for (int j = 0; j < U; j++) cc[j] = (k + j < m.y) ? (uint32_t)c[32 * (k + j)] : 0xFFFFu;
      // the rhs records (global memory) of the group's diagonal codes are
      // requested before any Hessian term is formed from shared memory
      double qx[U], qy[U], qz[U];
#pragma unroll
      for (int j = 0; j < U; j++) {
        qx[j] = qy[j] = qz[j] = 0.0;
        const uint32_t lt = cc[j] >> 4, a = (cc[j] >> 2) & 3u, bb = cc[j] & 3u;
        if (cc[j] != 0xFFFFu && a == bb && lt < (uint32_t)t.y) {
          const double4 q = st.rrec((uint32_t)gid[lt], a);
          qx[j] = q.x;
          qy[j] = q.y;
          qz[j] = q.z;
        }
      }
#pragma unroll
      for (int j = 0; j < U; j++) {
        const uint32_t lt = cc[j] >> 4, a = (cc[j] >> 2) & 3u, bb = cc[j] & 3u;
        if (cc[j] == 0xFFFFu || lt >= (uint32_t)t.y) continue;  // padding (the builder checks every code)
        acc_tet<R, V4>(sh[4 * lt + a], sh[4 * lt + bb], a == bb, g, b);
        r[0] += qx[j];
        r[1] += qy[j];
        r[2] += qz[j];
      }
    }
    cz_codes<S, CZ_UNROLL>(st, czcodes + m.w + lane, 0, m.z, b, dg ? r : nullptr);
    if (u.x >= 0) {
      st_block(vals, u.x, b);
#pragma unroll
      for (int q = 0; q < 9; q++) bad |= !isfinite((double)b[q]);
    }
    if (dg) {
      st_rhs(rhs, u.y, r);
      bad |= !(isfinite(r[0]) && isfinite(r[1]) && isfinite(r[2]));
    }
    int nw = 0;
    if (lane == 0) nw = atomicAdd(&next_slice, 1);
    w = __shfl_sync(0xffffffffu, nw, 0);
  }
  // no barrier at the end: each warp reports on its own
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(nonfinite, 1);
}

// ---- the fused row-tile kernel: tets computed in shared memory ---------------------
// As k_gather_tile, but the CTA computes the records of its tile's tets itself
// (tet_eval, the arithmetic of k_tet_unit) instead of copying them from the
// staging the tet kernel writes, so the tet records never reach global
// memory: no 256 B/tet store and no re-reads by the gathers.  A tet with
// vertices in several tiles is computed once per tile (about twice).  Shared
// memory per tet: the four {h_a, V} records (FP64 double4, or FP32-mixed
// float4) and the 12 FP64 rhs values; then the slice metadata, units and
// 16-bit tet codes of the tile.  The blocks are summed in the same order
// from the same values as in k_gather_tile: the results are bit-identical.
template <typename S, int MINB>
__global__ void __launch_bounds__(TILE_THREADS, MINB)
    k_tile_fused(const int4 *__restrict__ tiles, const int2 *__restrict__ trange, const int *__restrict__ ttet,
                 const int4 *__restrict__ meta, const int2 *__restrict__ unit, const uint16_t *__restrict__ tcodes,
                 const uint32_t *__restrict__ czcodes, S st, gargs<typename S::real> g,
                 const int4 *__restrict__ elem, const double4 *__restrict__ x0, const double4 *__restrict__ xc,
                 const double2 *__restrict__ va, icf_dprm P, double *__restrict__ vals, double *__restrict__ rhs,
                 int *__restrict__ nonfinite) {
  typedef typename S::real R;
  typedef typename S::rec V4;
  extern __shared__ __align__(16) unsigned char tile_smem[];
  __shared__ int next_slice;
  const int4 t = tiles[blockIdx.x];
  const int2 tr = trange[blockIdx.x];
  V4 *sh = reinterpret_cast<V4 *>(tile_smem);
  double *srhs = reinterpret_cast<double *>(sh + 4 * t.y);
  int4 *smeta = reinterpret_cast<int4 *>(srhs + 12 * t.y);
  int2 *sunit = reinterpret_cast<int2 *>(smeta + t.w);
  uint16_t *scode = reinterpret_cast<uint16_t *>(sunit + 32 * t.w);
  const int tid = threadIdx.x, nth = blockDim.x;
  // the tile's lists arrive by cp.async while the tets are computed
  for (int q = tid; q < t.w; q += nth) cp16(smeta + q, meta + t.z + q);
  for (int q = tid; q < 16 * t.w; q += nth) cp16(sunit + 2 * q, unit + 32 * (size_t)t.z + 2 * q);
  for (int q = tid; q < tr.y / 8; q += nth) cp16(scode + 8 * q, tcodes + tr.x + 8 * q);
  for (int k = tid; k < t.y; k += nth) {
    const int e = __ldg(ttet + t.x + k);
    icf_tet_out o;
    tet_eval(e, elem, x0, xc, va, P, o);
#pragma unroll
    for (int a = 0; a < 4; a++) {
      V4 r;
      r.x = (R)o.h[a][0];
      r.y = (R)o.h[a][1];
      r.z = (R)o.h[a][2];
      r.w = (R)o.V;
      sh[4 * k + a] = r;
#pragma unroll
      for (int c = 0; c < 3; c++) srhs[12 * k + 3 * a + c] = o.r[a][c];
    }
  }
  if (tid == 0) next_slice = nth >> 5;
  cp_wait_all();
  __syncthreads();
  const int lane = tid & 31;
  bool bad = false;
  int w = tid >> 5;
  while (w < t.w) {
    const int4 m = smeta[w];
    const int2 u = sunit[32 * w + lane];
    const bool dg = u.y >= 0;
    const uint16_t *c = scode + (m.x - tr.x) + lane;
    R b[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double r[3] = {0, 0, 0};
    for (int k = 0; k < m.y; k++) {
      const uint32_t cc = (uint32_t)c[32 * k];
      const uint32_t lt = cc >> 4, a = (cc >> 2) & 3u, bb = cc & 3u;
      if (cc == 0xFFFFu || lt >= (uint32_t)t.y) continue;  // padding (the builder checks every code)
      acc_tet<R, V4>(sh[4 * lt + a], sh[4 * lt + bb], a == bb, g, b);
      if (a == bb) {
        const double *q = srhs + 12 * lt + 3 * a;
        r[0] += q[0];
        r[1] += q[1];
        r[2] += q[2];
      }
    }
    cz_codes<S, CZ_UNROLL>(st, czcodes + m.w + lane, 0, m.z, b, dg ? r : nullptr);
    if (u.x >= 0) {
      st_block(vals, u.x, b);
#pragma unroll
      for (int q = 0; q < 9; q++) bad |= !isfinite((double)b[q]);
    }
    if (dg) {
      st_rhs(rhs, u.y, r);
      bad |= !(isfinite(r[0]) && isfinite(r[1]) && isfinite(r[2]));
    }
    int nw = 0;
    if (lane == 0) nw = atomicAdd(&next_slice, 1);
    w = __shfl_sync(0xffffffffu, nw, 0);
  }
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(nonfinite, 1);
}

#define OFFV(MB, U)                                                                                   \
  {"reg minb" #MB " u" #U, k_gather_off<fp64, MB, U>, k_gather_off<fp32mixed, MB, U>,                \
   k_gather_off_c<fp64, false, MB, U>, k_gather_off_c<fp32mixed, true, MB, U>, 0, false}
#define OFFN(MB, U)                                                                                   \
  {"natural minb" #MB " u" #U, k_gather_off_nat<fp64, MB, U>, k_gather_off_nat<fp32mixed, MB, U>,   \
   k_gather_off_c<fp64, false, MB, U>, k_gather_off_c<fp32mixed, true, MB, U>, 0, true}
#define OFFS(MB, U)                                                                                   \
  {"stream minb" #MB " u" #U, k_gather_off_cs<fp64, MB, U>, k_gather_off_cs<fp32mixed, MB, U>,      \
   k_gather_off_c<fp64, false, MB, U>, k_gather_off_c<fp32mixed, true, MB, U>, 0, false}
#define OFFP(MB, U)                                                                                   \
  {"pipe minb" #MB " u" #U, k_gather_off_pipe<fp64, MB, U>, k_gather_off_pipe<fp32mixed, MB, U>,     \
   k_gather_off_c<fp64, false, MB, U>, k_gather_off_c<fp32mixed, true, MB, U>, MB, false}
#define DIAGV(L, MB, U)                                                                               \
  {"reg L" #L " minb" #MB " u" #U, L, k_gather_diag<fp64, L, MB, U>, k_gather_diag<fp32mixed, L, MB, U>, \
   k_gather_diag_c<fp64, false, L, MB, U>, k_gather_diag_c<fp32mixed, true, L, MB, U>, 0}
#define DIAGP(L, MB, U)                                                                               \
  {"pipe L" #L " minb" #MB " u" #U, L, k_gather_diag_pipe<fp64, L, MB, U>,                           \
   k_gather_diag_pipe<fp32mixed, L, MB, U>, k_gather_diag_c<fp64, false, L, MB, U>,                  \
   k_gather_diag_c<fp32mixed, true, L, MB, U>, MB}
const off_variant OFF_VARIANTS[] = {OFFV(4, 4), OFFV(3, 2), OFFV(2, 4), OFFV(4, 2), OFFP(4, 2), OFFP(3, 4),
                                    OFFN(4, 2), OFFN(4, 4), OFFN(3, 2), OFFS(4, 2), OFFS(4, 4)};
const diag_variant DIAG_VARIANTS[] = {DIAGV(4, 4, 4), DIAGV(2, 3, 4), DIAGV(4, 2, 4), DIAGV(8, 4, 2),
                                      DIAGV(2, 4, 2), DIAGP(4, 4, 2), DIAGP(8, 4, 2)};
#undef OFFV
#undef OFFN
#undef OFFS
#undef OFFP
#undef DIAGV
#undef DIAGP
constexpr int N_OFF = sizeof(OFF_VARIANTS) / sizeof(OFF_VARIANTS[0]);
constexpr int N_DIAG = sizeof(DIAG_VARIANTS) / sizeof(DIAG_VARIANTS[0]);

fp32mixed mixed_views(const icf_ctx *ctx, const double4 *es, const double *cs) {
  fp32mixed m;
  m.esr = es;
  m.es32 = reinterpret_cast<const float4 *>(es + 4 * (size_t)ctx->n_elem);
  m.csr = cs;
  m.cs32 = reinterpret_cast<const float *>(cs + 12 * (size_t)ctx->n_cz);
  return m;
}

}  // namespace

// Shared memory of the tiled gather for the largest tile (outside any capture).
int icf_gather_tile_setup(icf_ctx *ctx) {
  const icf_tiles &T = ctx->tiles;
  ICF_CUDA(ctx, cudaFuncSetAttribute(k_tile_fused<fp32mixed, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)T.smemf32));
  ICF_CUDA(ctx, cudaFuncSetAttribute(k_tile_fused<fp64, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)T.smemf64));
  ICF_CUDA(ctx, cudaFuncSetAttribute(k_gather_tile<fp32mixed, 4, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)T.smem32));
  ICF_CUDA(ctx, cudaFuncSetAttribute(k_gather_tile<fp64, 3, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)T.smem64));
  return ICF_OK;
}

int icf_launch_gather_tile(icf_ctx *ctx, const double4 *es, const double *cs, double sc, double mc, double lam,
                           double mu, double *vals, double *rhs, cudaStream_t s) {
  const icf_tiles &T = ctx->tiles;
  if (T.n_tiles == 0) return ICF_OK;
  if (ctx->precision == ICF_FP32_MIXED) {
    const gargs<float> g{(float)sc, (float)mc, (float)lam, (float)mu};
    k_gather_tile<fp32mixed, 4, 2><<<T.n_tiles, TILE_THREADS, T.smem32, s>>>(
        T.tiles, T.trange, T.ttet, T.meta, T.unit, T.tcodes, T.czcodes, mixed_views(ctx, es, cs), g, vals, rhs,
        ctx->d_counts + 4);
  } else {
    fp64 st;
    st.es = es;
    st.cs = cs;
    const gargs<double> g{sc, mc, lam, mu};
    k_gather_tile<fp64, 3, 2><<<T.n_tiles, TILE_THREADS, T.smem64, s>>>(T.tiles, T.trange, T.ttet, T.meta, T.unit,
                                                               T.tcodes, T.czcodes, st, g, vals, rhs,
                                                               ctx->d_counts + 4);
  }
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}

int icf_launch_tile_fused(icf_ctx *ctx, const double4 *xc, const double2 *va, const double *cs, double sc,
                          double mc, double *vals, double *rhs, cudaStream_t s) {
  const icf_tiles &T = ctx->tiles;
  if (T.n_tiles == 0) return ICF_OK;
  const icf_dprm P = icf_make_dprm(ctx);
  if (ctx->precision == ICF_FP32_MIXED) {
    const gargs<float> g{(float)sc, (float)mc, (float)P.lam, (float)P.mu};
    k_tile_fused<fp32mixed, 2><<<T.n_tiles, TILE_THREADS, T.smemf32, s>>>(
        T.tiles, T.trange, T.ttet, T.meta, T.unit, T.tcodes, T.czcodes, mixed_views(ctx, ctx->d_es, cs), g,
        ctx->d_elem, ctx->d_x0, xc, va, P, vals, rhs, ctx->d_counts + 4);
  } else {
    fp64 st;
    st.es = nullptr;
    st.cs = cs;
    const gargs<double> g{sc, mc, P.lam, P.mu};
    k_tile_fused<fp64, 2><<<T.n_tiles, TILE_THREADS, T.smemf64, s>>>(
        T.tiles, T.trange, T.ttet, T.meta, T.unit, T.tcodes, T.czcodes, st, g, ctx->d_elem, ctx->d_x0, xc, va, P,
        vals, rhs, ctx->d_counts + 4);
  }
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}

int icf_gather_variants(int kind) { return kind == 0 ? N_OFF : N_DIAG; }
const char *icf_gather_variant_name(int kind, int v) {
  return kind == 0 ? OFF_VARIANTS[v].name : DIAG_VARIANTS[v].name;
}
int icf_gather_variant_lanes(int v) { return DIAG_VARIANTS[v].lanes; }
bool icf_gather_variant_natural(int v) { return OFF_VARIANTS[v].natural; }

int icf_launch_gather_off(icf_ctx *ctx, const icf_sell &S, int variant, const double4 *es, const double *cs,
                          double sc, double mc, double lam, double mu, double *vals, cudaStream_t s) {
  if (S.n_slices == 0) return ICF_OK;
  if (variant < 0 || variant >= N_OFF) variant = 0;
  unsigned grid = icf_blocks(32LL * S.n_slices, 256);
  const int pm = OFF_VARIANTS[variant].persistent_minb;
  if (pm > 0 && ctx->layout == ICF_LAYOUT_RECORDS && grid > (unsigned)(ctx->n_sm * pm)) grid = ctx->n_sm * pm;
  const char *stage = static_cast<const char *>(ctx->d_stage_off);
  if (ctx->layout == ICF_LAYOUT_CONTRIB && ctx->precision == ICF_FP32_MIXED) {
    const gargs<float> g{(float)sc, (float)mc, (float)lam, (float)mu};
    OFF_VARIANTS[variant].c32<<<grid, 256, 0, s>>>(S.n_slices, S.meta, S.unit, S.codes, stage,
                                                  mixed_views(ctx, es, cs), g, vals);
  } else if (ctx->layout == ICF_LAYOUT_CONTRIB) {
    fp64 st;
    st.es = es;
    st.cs = cs;
    const gargs<double> g{sc, mc, lam, mu};
    OFF_VARIANTS[variant].c64<<<grid, 256, 0, s>>>(S.n_slices, S.meta, S.unit, S.codes, stage, st, g, vals);
  } else if (ctx->precision == ICF_FP32_MIXED) {
    const gargs<float> g{(float)sc, (float)mc, (float)lam, (float)mu};
    OFF_VARIANTS[variant].f32<<<grid, 256, 0, s>>>(S.n_slices, S.meta, S.unit, S.codes, mixed_views(ctx, es, cs),
                                                  g, vals);
  } else {
    fp64 st;
    st.es = es;
    st.cs = cs;
    const gargs<double> g{sc, mc, lam, mu};
    OFF_VARIANTS[variant].f64<<<grid, 256, 0, s>>>(S.n_slices, S.meta, S.unit, S.codes, st, g, vals);
  }
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}

int icf_launch_gather_diag(icf_ctx *ctx, const icf_sell &S, int variant, const double4 *es, const double *cs,
                           double sc, double mc, double lam, double mu, double *vals, double *rhs, cudaStream_t s) {
  if (S.n_slices == 0) return ICF_OK;
  if (variant < 0 || variant >= N_DIAG || DIAG_VARIANTS[variant].lanes != S.lanes) {
    // the lists were built for S.lanes: take the first variant that reads them
    variant = -1;
    for (int v = 0; v < N_DIAG && variant < 0; v++)
      if (DIAG_VARIANTS[v].lanes == S.lanes) variant = v;
    if (variant < 0) return icf_fail(ctx, ICF_ERR_STATE, "no diagonal gather for this list layout");
  }
  unsigned grid = icf_blocks(32LL * S.n_slices, 256);
  const int pm = DIAG_VARIANTS[variant].persistent_minb;
  if (pm > 0 && ctx->layout == ICF_LAYOUT_RECORDS && grid > (unsigned)(ctx->n_sm * pm)) grid = ctx->n_sm * pm;
  const char *stage = static_cast<const char *>(ctx->d_stage_diag);
  if (ctx->layout == ICF_LAYOUT_CONTRIB && ctx->precision == ICF_FP32_MIXED) {
    const gargs<float> g{(float)sc, (float)mc, (float)lam, (float)mu};
    DIAG_VARIANTS[variant].c32<<<grid, 256, 0, s>>>(S.n_slices, S.meta, S.unit, S.codes, stage,
                                                   mixed_views(ctx, es, cs), g, vals, rhs, ctx->d_counts + 4);
  } else if (ctx->layout == ICF_LAYOUT_CONTRIB) {
    fp64 st;
    st.es = es;
    st.cs = cs;
    const gargs<double> g{sc, mc, lam, mu};
    DIAG_VARIANTS[variant].c64<<<grid, 256, 0, s>>>(S.n_slices, S.meta, S.unit, S.codes, stage, st, g, vals,
                                                   rhs, ctx->d_counts + 4);
  } else if (ctx->precision == ICF_FP32_MIXED) {
    const gargs<float> g{(float)sc, (float)mc, (float)lam, (float)mu};
    DIAG_VARIANTS[variant].f32<<<grid, 256, 0, s>>>(S.n_slices, S.meta, S.unit, S.codes,
                                                   mixed_views(ctx, es, cs), g, vals, rhs, ctx->d_counts + 4);
  } else {
    fp64 st;
    st.es = es;
    st.cs = cs;
    const gargs<double> g{sc, mc, lam, mu};
    DIAG_VARIANTS[variant].f64<<<grid, 256, 0, s>>>(S.n_slices, S.meta, S.unit, S.codes, st, g, vals, rhs,
                                                   ctx->d_counts + 4);
  }
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}
