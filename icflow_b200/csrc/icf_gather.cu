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
// iteration, loads through registers or through cp.async into shared memory,
// lanes per row).  They compute the same sums in the same order; the
// autotuner (icf_tune.cu) times them on the model at hand and keeps the
// fastest.
#include <cstdint>

#include "icf_internal.cuh"

namespace {

__device__ __forceinline__ int sym_pair(int i, int j) {
  // (0,0)0 (0,1)1 (0,2)2 (1,1)3 (1,2)4 (2,2)5
  const int lo = i < j ? i : j, hi = i < j ? j : i;
  return lo == 0 ? hi : (lo == 1 ? 2 + hi : 5);
}

struct gargs {
  double sc, mc, lam, mu;
};

// LHS_ab = stiffCoeff Df_ab + massCoeff M_ab rebuilt from the staging records
// {h_a, V} and {h_b, V} of one tet (k_tet_unit):
//   Df_ab = V (lam h_a h_b^T + mu h_b h_a^T + mu (h_a.h_b) I),
//   M_ab = rho/20 (1 + delta_ab) V I.
// A zero record (a padding code) adds nothing.
__device__ __forceinline__ void acc_tet(const double4 &A, const double4 &B, bool diag, const gargs &g,
                                        double b[9]) {
  const double V = A.w;
  const double ha[3] = {A.x, A.y, A.z}, hb[3] = {B.x, B.y, B.z};
  const double dot = ha[0] * hb[0] + ha[1] * hb[1] + ha[2] * hb[2];
  const double c1 = g.sc * V * g.lam, c2 = g.sc * V * g.mu;
  const double cd = c2 * dot + g.mc * V * (diag ? 2.0 : 1.0);
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int l = 0; l < 3; l++) b[3 * k + l] += c1 * ha[k] * hb[l] + c2 * hb[k] * ha[l] + (k == l ? cd : 0.0);
}

__device__ __forceinline__ void tet_code(uint32_t code, uint32_t &e, uint32_t &a, uint32_t &b) {
  e = (code >> 4) & 0x3FFFFFFu;
  a = (code >> 2) & 3u;
  b = code & 3u;
}

// Contribution of one CZ code: +-Kt[a mod 3][b mod 3] (symmetric 3x3) and,
// for a diagonal block, -+rt[a mod 3].
__device__ __forceinline__ void add_cz(uint32_t code, const double *__restrict__ cs, double b[9],
                                       double *r) {
  const uint32_t c = (code >> 6) & 0xFFFFFFu, a = (code >> 3) & 7u, bb = code & 7u;
  const double *S = cs + (size_t)c * ICF_CZ_STAGE;
  const int ia = a % 3, ib = bb % 3;
  const double sg = ((a < 3) == (bb < 3)) ? 1.0 : -1.0;
  const double2 *K2 = reinterpret_cast<const double2 *>(S + 6 * sym_pair(ia, ib));
  const double2 k01 = __ldg(K2), k23 = __ldg(K2 + 1), k45 = __ldg(K2 + 2);
  b[0] += sg * k01.x; b[1] += sg * k01.y; b[2] += sg * k23.x;
  b[3] += sg * k01.y; b[4] += sg * k23.y; b[5] += sg * k45.x;
  b[6] += sg * k23.x; b[7] += sg * k45.x; b[8] += sg * k45.y;
  if (r != nullptr) {
    const double sa = (a < 3) ? -1.0 : 1.0;
    r[0] += sa * __ldg(S + 36 + 3 * ia + 0);
    r[1] += sa * __ldg(S + 36 + 3 * ia + 1);
    r[2] += sa * __ldg(S + 36 + 3 * ia + 2);
  }
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_rec(double4 *smem, const double4 *gmem) {
  cp_async16(smem, gmem);
  cp_async16(reinterpret_cast<char *>(smem) + 16, reinterpret_cast<const char *>(gmem) + 16);
}

// ---- off-diagonal blocks: one lane per block --------------------------------

// Records through registers: U codes per iteration, their 2U records loaded
// before any is used.
template <int MINB, int U>
__global__ void __launch_bounds__(256, MINB)
    k_gather_off_reg(int n_slices, const int4 *__restrict__ meta, const int2 *__restrict__ unit,
                     const uint32_t *__restrict__ codes, const double4 *__restrict__ es,
                     const double *__restrict__ cs, gargs g, double *__restrict__ vals) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= n_slices) return;
  const int4 m = meta[w];
  const uint32_t *c = codes + m.x + lane;
  double b[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int k = 0; k < m.y; k += U) {
    uint32_t cc[U];
#pragma unroll
    for (int j = 0; j < U; j++) cc[j] = (k + j < m.y) ? __ldg(c + 32 * (k + j)) : ICF_CODE_PAD;
    double4 A[U], B[U];
#pragma unroll
    for (int j = 0; j < U; j++) {
      A[j] = B[j] = make_double4(0, 0, 0, 0);
      if (cc[j] != ICF_CODE_PAD) {
        uint32_t e, a, bb;
        tet_code(cc[j], e, a, bb);
        A[j] = es[8 * (size_t)e + a];
        B[j] = es[8 * (size_t)e + bb];
      }
    }
#pragma unroll
    for (int j = 0; j < U; j++) acc_tet(A[j], B[j], false, g, b);
  }
  for (int k = m.y; k < m.y + m.z; k++) {
    const uint32_t c0 = __ldg(c + 32 * k);
    if (c0 != ICF_CODE_PAD) add_cz(c0, cs, b, nullptr);
  }
  const int2 u = unit[32 * w + lane];
  if (u.x < 0) return;
  double *o = vals + 9 * (size_t)u.x;
#pragma unroll
  for (int q = 0; q < 9; q++) o[q] = b[q];
}

// Records through shared memory: the 2U records of an iteration are copied
// with cp.async (no registers held while they are in flight), then read back
// conflict-free (record j of the 32 lanes is contiguous).
template <int T, int U>
__global__ void __launch_bounds__(T)
    k_gather_off_async(int n_slices, const int4 *__restrict__ meta, const int2 *__restrict__ unit,
                       const uint32_t *__restrict__ codes, const double4 *__restrict__ es,
                       const double *__restrict__ cs, gargs g, double *__restrict__ vals) {
  extern __shared__ double4 sm_rec[];
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= n_slices) return;
  double4 *my = sm_rec + (size_t)(threadIdx.x >> 5) * (2 * U * 32);
  const int4 m = meta[w];
  const uint32_t *c = codes + m.x + lane;
  double b[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int k = 0; k < m.y; k += U) {
    uint32_t cc[U];
#pragma unroll
    for (int j = 0; j < U; j++) cc[j] = (k + j < m.y) ? __ldg(c + 32 * (k + j)) : ICF_CODE_PAD;
#pragma unroll
    for (int j = 0; j < U; j++)
      if (cc[j] != ICF_CODE_PAD) {
        uint32_t e, a, bb;
        tet_code(cc[j], e, a, bb);
        cp_async_rec(my + (2 * j) * 32 + lane, es + 8 * (size_t)e + a);
        cp_async_rec(my + (2 * j + 1) * 32 + lane, es + 8 * (size_t)e + bb);
      }
    cp_async_wait_all();
#pragma unroll
    for (int j = 0; j < U; j++)
      if (cc[j] != ICF_CODE_PAD) acc_tet(my[(2 * j) * 32 + lane], my[(2 * j + 1) * 32 + lane], false, g, b);
  }
  for (int k = m.y; k < m.y + m.z; k++) {
    const uint32_t c0 = __ldg(c + 32 * k);
    if (c0 != ICF_CODE_PAD) add_cz(c0, cs, b, nullptr);
  }
  const int2 u = unit[32 * w + lane];
  if (u.x < 0) return;
  double *o = vals + 9 * (size_t)u.x;
#pragma unroll
  for (int q = 0; q < 9; q++) o[q] = b[q];
}

// ---- diagonal blocks and rhs rows: L lanes per row --------------------------
// Every code of a diagonal block has a == b: one {h, V} record for the block
// and one {rhs, 0} record for the row.  The L partial sums are combined by a
// fixed shuffle tree.
template <int L>
__device__ __forceinline__ void diag_finish(int w, int lane, const int2 *__restrict__ unit, double b[9],
                                            double r[3], double *__restrict__ vals,
                                            double *__restrict__ rhs) {
#pragma unroll
  for (int o = 1; o < L; o <<= 1) {
#pragma unroll
    for (int q = 0; q < 9; q++) b[q] += __shfl_xor_sync(0xffffffffu, b[q], o);
#pragma unroll
    for (int q = 0; q < 3; q++) r[q] += __shfl_xor_sync(0xffffffffu, r[q], o);
  }
  const int sub = lane % L;
  const int2 u = unit[(32 / L) * w + lane / L];
  const bool wb = (sub == 0), wr = (L == 1) ? true : (sub == 1);
  if (wb && u.x >= 0) {
    double *o = vals + 9 * (size_t)u.x;
#pragma unroll
    for (int q = 0; q < 9; q++) o[q] = b[q];
  }
  if (wr && u.y >= 0) {
    rhs[3 * (size_t)u.y + 0] = r[0];
    rhs[3 * (size_t)u.y + 1] = r[1];
    rhs[3 * (size_t)u.y + 2] = r[2];
  }
}

template <int L, int MINB, int U>
__global__ void __launch_bounds__(256, MINB)
    k_gather_diag_reg(int n_slices, const int4 *__restrict__ meta, const int2 *__restrict__ unit,
                      const uint32_t *__restrict__ codes, const double4 *__restrict__ es,
                      const double *__restrict__ cs, gargs g, double *__restrict__ vals,
                      double *__restrict__ rhs) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= n_slices) return;
  const int4 m = meta[w];
  const uint32_t *c = codes + m.x + lane;
  double b[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, r[3] = {0, 0, 0};
  for (int k = 0; k < m.y; k += U) {
    uint32_t cc[U];
#pragma unroll
    for (int j = 0; j < U; j++) cc[j] = (k + j < m.y) ? __ldg(c + 32 * (k + j)) : ICF_CODE_PAD;
    double4 A[U], R[U];
#pragma unroll
    for (int j = 0; j < U; j++) {
      A[j] = R[j] = make_double4(0, 0, 0, 0);
      if (cc[j] != ICF_CODE_PAD) {
        uint32_t e, a, bb;
        tet_code(cc[j], e, a, bb);
        A[j] = es[8 * (size_t)e + a];
        R[j] = es[8 * (size_t)e + 4 + a];
      }
    }
#pragma unroll
    for (int j = 0; j < U; j++) {
      acc_tet(A[j], A[j], true, g, b);
      r[0] += R[j].x;
      r[1] += R[j].y;
      r[2] += R[j].z;
    }
  }
  for (int k = m.y; k < m.y + m.z; k++) {
    const uint32_t c0 = __ldg(c + 32 * k);
    if (c0 != ICF_CODE_PAD) add_cz(c0, cs, b, r);
  }
  diag_finish<L>(w, lane, unit, b, r, vals, rhs);
}

template <int T, int L, int U>
__global__ void __launch_bounds__(T)
    k_gather_diag_async(int n_slices, const int4 *__restrict__ meta, const int2 *__restrict__ unit,
                        const uint32_t *__restrict__ codes, const double4 *__restrict__ es,
                        const double *__restrict__ cs, gargs g, double *__restrict__ vals,
                        double *__restrict__ rhs) {
  extern __shared__ double4 sm_rec[];
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= n_slices) return;
  double4 *my = sm_rec + (size_t)(threadIdx.x >> 5) * (2 * U * 32);
  const int4 m = meta[w];
  const uint32_t *c = codes + m.x + lane;
  double b[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, r[3] = {0, 0, 0};
  for (int k = 0; k < m.y; k += U) {
    uint32_t cc[U];
#pragma unroll
    for (int j = 0; j < U; j++) cc[j] = (k + j < m.y) ? __ldg(c + 32 * (k + j)) : ICF_CODE_PAD;
#pragma unroll
    for (int j = 0; j < U; j++)
      if (cc[j] != ICF_CODE_PAD) {
        uint32_t e, a, bb;
        tet_code(cc[j], e, a, bb);
        cp_async_rec(my + (2 * j) * 32 + lane, es + 8 * (size_t)e + a);
        cp_async_rec(my + (2 * j + 1) * 32 + lane, es + 8 * (size_t)e + 4 + a);
      }
    cp_async_wait_all();
#pragma unroll
    for (int j = 0; j < U; j++)
      if (cc[j] != ICF_CODE_PAD) {
        const double4 A = my[(2 * j) * 32 + lane], R = my[(2 * j + 1) * 32 + lane];
        acc_tet(A, A, true, g, b);
        r[0] += R.x;
        r[1] += R.y;
        r[2] += R.z;
      }
  }
  for (int k = m.y; k < m.y + m.z; k++) {
    const uint32_t c0 = __ldg(c + 32 * k);
    if (c0 != ICF_CODE_PAD) add_cz(c0, cs, b, r);
  }
  diag_finish<L>(w, lane, unit, b, r, vals, rhs);
}

// ---- variant tables ---------------------------------------------------------
typedef void (*off_fn)(int, const int4 *, const int2 *, const uint32_t *, const double4 *, const double *, gargs,
                       double *);
typedef void (*diag_fn)(int, const int4 *, const int2 *, const uint32_t *, const double4 *, const double *,
                        gargs, double *, double *);

struct off_variant {
  const char *name;
  off_fn fn;
  int threads;
  int smem;  // dynamic shared memory per block
};
struct diag_variant {
  const char *name;
  diag_fn fn;
  int threads, smem, lanes;
};

const off_variant OFF_VARIANTS[] = {
    {"reg minb4 u4", k_gather_off_reg<4, 4>, 256, 0},
    {"reg minb2 u4", k_gather_off_reg<2, 4>, 256, 0},
    {"reg minb3 u2", k_gather_off_reg<3, 2>, 256, 0},
    {"async t128 u4", k_gather_off_async<128, 4>, 128, 4 * 2 * 4 * 32 * 32},
    {"async t128 u8", k_gather_off_async<128, 8>, 128, 4 * 2 * 8 * 32 * 32},
    {"async t256 u4", k_gather_off_async<256, 4>, 256, 8 * 2 * 4 * 32 * 32},
};
const diag_variant DIAG_VARIANTS[] = {
    {"reg L4 minb4 u4", k_gather_diag_reg<4, 4, 4>, 256, 0, 4},
    {"reg L4 minb2 u4", k_gather_diag_reg<4, 2, 4>, 256, 0, 4},
    {"reg L2 minb3 u4", k_gather_diag_reg<2, 3, 4>, 256, 0, 2},
    {"reg L8 minb4 u2", k_gather_diag_reg<8, 4, 2>, 256, 0, 8},
    {"async t128 L4 u4", k_gather_diag_async<128, 4, 4>, 128, 4 * 2 * 4 * 32 * 32, 4},
    {"async t128 L2 u8", k_gather_diag_async<128, 2, 8>, 128, 4 * 2 * 8 * 32 * 32, 2},
};
constexpr int N_OFF = sizeof(OFF_VARIANTS) / sizeof(OFF_VARIANTS[0]);
constexpr int N_DIAG = sizeof(DIAG_VARIANTS) / sizeof(DIAG_VARIANTS[0]);

bool g_attrs_set[64] = {false};

}  // namespace

int icf_gather_variants(int kind) { return kind == 0 ? N_OFF : N_DIAG; }
const char *icf_gather_variant_name(int kind, int v) {
  return kind == 0 ? OFF_VARIANTS[v].name : DIAG_VARIANTS[v].name;
}
int icf_gather_variant_lanes(int v) { return DIAG_VARIANTS[v].lanes; }

// Opts the shared-memory variants into more than 48 KB of dynamic shared
// memory (once per device).
static int set_smem_attrs(icf_ctx *ctx) {
  if (ctx->device < 0 || ctx->device >= 64 || g_attrs_set[ctx->device]) return ICF_OK;
  for (int v = 0; v < N_OFF; v++)
    if (OFF_VARIANTS[v].smem > 0)
      ICF_CUDA(ctx, cudaFuncSetAttribute(reinterpret_cast<const void *>(OFF_VARIANTS[v].fn),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, OFF_VARIANTS[v].smem));
  for (int v = 0; v < N_DIAG; v++)
    if (DIAG_VARIANTS[v].smem > 0)
      ICF_CUDA(ctx, cudaFuncSetAttribute(reinterpret_cast<const void *>(DIAG_VARIANTS[v].fn),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, DIAG_VARIANTS[v].smem));
  g_attrs_set[ctx->device] = true;
  return ICF_OK;
}

int icf_launch_gather_off(icf_ctx *ctx, int variant, const double4 *es, const double *cs, double sc, double mc,
                          double lam, double mu, double *vals, cudaStream_t s) {
  const icf_sell &S = ctx->sell_off;
  if (S.n_slices == 0) return ICF_OK;
  if (variant < 0 || variant >= N_OFF) variant = 0;
  if (set_smem_attrs(ctx)) return ICF_ERR_CUDA;
  const off_variant &V = OFF_VARIANTS[variant];
  const gargs g{sc, mc, lam, mu};
  V.fn<<<icf_blocks(32LL * S.n_slices, V.threads), V.threads, V.smem, s>>>(S.n_slices, S.meta, S.unit, S.codes,
                                                                          es, cs, g, vals);
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}

int icf_launch_gather_diag(icf_ctx *ctx, int variant, const double4 *es, const double *cs, double sc,
                           double mc, double lam, double mu, double *vals, double *rhs, cudaStream_t s) {
  const icf_sell &S = ctx->sell_diag;
  if (S.n_slices == 0) return ICF_OK;
  if (variant < 0 || variant >= N_DIAG || DIAG_VARIANTS[variant].lanes != S.lanes) {
    // the lists were built for S.lanes: take the first variant that reads them
    variant = -1;
    for (int v = 0; v < N_DIAG && variant < 0; v++)
      if (DIAG_VARIANTS[v].lanes == S.lanes) variant = v;
    if (variant < 0) return icf_fail(ctx, ICF_ERR_STATE, "no diagonal gather for this list layout");
  }
  if (set_smem_attrs(ctx)) return ICF_ERR_CUDA;
  const diag_variant &V = DIAG_VARIANTS[variant];
  const gargs g{sc, mc, lam, mu};
  V.fn<<<icf_blocks(32LL * S.n_slices, V.threads), V.threads, V.smem, s>>>(S.n_slices, S.meta, S.unit, S.codes,
                                                                          es, cs, g, vals, rhs);
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}
