// icf_solve.cu -- the Newton linear solve on the device.
//
// The reference copies the upper-triangular BCSR matrix and the rhs to the
// host every Newton iteration and solves them with MKL PARDISO (symmetric,
// mtype -2, BSR 3x3; LinearSystem.cs:45-64, PardisoLoader2/dllmain.cpp:30-79).
// Here the system stays where it was assembled and is solved by
// the minimal residual method (MINRES: the matrix is symmetric but, with
// softening cohesive zones, may be indefinite, as PARDISO's mtype -2 allows)
// with a block-Jacobi (3x3) preconditioner, positive definite as MINRES needs
// (a row whose diagonal block is indefinite uses |S|^-1 of the block's
// symmetric part):
//   - A x uses the stored upper blocks directly and their transposes through
//     a per-structure index of the lower blocks (row = column of the upper
//     block), four lanes per row and a fixed shuffle tree, so every product
//     is deterministic;
//   - dot products reduce per block and then in one block, in a fixed order;
//   - the MINRES scalars and plane rotations live on the device; the host
//     reads the residual estimate every few iterations only to stop.
// The solution stays on the device for icf_apply_dx (du += dx, the
// reference's _XtoDU, ImplicitModel3.cs:247-256).
#include <cub/cub.cuh>

#include <cstdio>

#include <cmath>
#include <string>

#include "icf_internal.cuh"

namespace {

constexpr int RED_BLOCKS = 296;  // two blocks per SM for the reductions

// transposed (lower) blocks: key (col << 32 | row) of every off-diagonal slot
__global__ void k_lower_keys(int nnz, const unsigned long long *__restrict__ mkeys,
                             unsigned long long *__restrict__ key, int *__restrict__ slot) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nnz) return;
  const unsigned long long k = mkeys[s];
  const unsigned long long r = k >> 32, c = k & 0xffffffffull;
  key[s] = (r == c) ? ~0ull : (c << 32 | r);
  slot[s] = s;
}

__global__ void k_lower_rows(int N, int n, const unsigned long long *__restrict__ key, int *__restrict__ lrows,
                             int *__restrict__ lcols) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r <= N) {
    const unsigned long long target = (unsigned long long)r << 32;
    int lo = 0, hi = n;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (key[mid] < target) lo = mid + 1;
      else hi = mid;
    }
    lrows[r] = lo;
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (key[i] != ~0ull) lcols[i] = (int)(key[i] & 0xffffffffull);
}

// |S|^-1 for a symmetric 3x3 block S = V diag(l) V^T: V diag(1 / |l|) V^T,
// the eigenvalues by cyclic Jacobi rotations (Golub & Van Loan, Matrix
// Computations, section 8.5), |l| floored at 1e-14 of the largest.  Returns
// false when S is zero or not finite.
__device__ bool abs_inverse_sym3(const double S[9], double *o) {
  double a[3][3], v[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      a[i][j] = S[3 * i + j];
      v[i][j] = i == j ? 1.0 : 0.0;
    }
  for (int sweep = 0; sweep < 10; sweep++) {
    const double off = fabs(a[0][1]) + fabs(a[0][2]) + fabs(a[1][2]);
    const double dia = fabs(a[0][0]) + fabs(a[1][1]) + fabs(a[2][2]);
    if (!(off > 1e-300) || off <= 1e-18 * dia) break;
    for (int p = 0; p < 2; p++)
      for (int q = p + 1; q < 3; q++) {
        if (a[p][q] == 0.0) continue;
        const double th = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
        const double t = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
        // A <- J^T A J, V <- V J with J the rotation in the (p, q) plane
        for (int k = 0; k < 3; k++) {
          const double akp = a[k][p], akq = a[k][q];
          a[k][p] = c * akp - sn * akq;
          a[k][q] = sn * akp + c * akq;
        }
        for (int k = 0; k < 3; k++) {
          const double apk = a[p][k], aqk = a[q][k];
          a[p][k] = c * apk - sn * aqk;
          a[q][k] = sn * apk + c * aqk;
        }
        for (int k = 0; k < 3; k++) {
          const double vkp = v[k][p], vkq = v[k][q];
          v[k][p] = c * vkp - sn * vkq;
          v[k][q] = sn * vkp + c * vkq;
        }
      }
  }
  double l[3], lmax = 0;
  for (int i = 0; i < 3; i++) {
    l[i] = fabs(a[i][i]);
    lmax = fmax(lmax, l[i]);
  }
  if (!(lmax > 0) || !isfinite(lmax)) return false;
  for (int i = 0; i < 3; i++) l[i] = 1.0 / fmax(l[i], 1e-14 * lmax);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) o[3 * i + j] = v[i][0] * l[0] * v[j][0] + v[i][1] * l[1] * v[j][1] + v[i][2] * l[2] * v[j][2];
  return true;
}

// The preconditioner of each row: the inverse of its diagonal block (the
// first block of its row) when the block is positive definite; otherwise
// (softening cohesive zones can make it indefinite) |S|^-1 of its symmetric
// part S, which keeps the preconditioner positive definite as MINRES needs.
// bad: bit 0 a zero or non-finite block; count[0]: blocks replaced by |S|^-1.
__global__ void k_dinv(int N, const int *__restrict__ rows, const double *__restrict__ vals,
                       double *__restrict__ dinv, int *__restrict__ bad) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= N) return;
  const double *a = vals + 9 * (size_t)rows[r];
  const double c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8], c02 = a[3] * a[7] - a[4] * a[6];
  const double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
  double *o = dinv + 9 * (size_t)r;
  const double m2 = a[0] * a[4] - 0.25 * (a[1] + a[3]) * (a[1] + a[3]);
  if (!(a[0] > 0 && m2 > 0 && det > 0) || !isfinite(det)) {
    double S[9];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) S[3 * i + j] = 0.5 * (a[3 * i + j] + a[3 * j + i]);
    if (!abs_inverse_sym3(S, o)) {
      atomicOr(bad, 1);
      for (int k = 0; k < 9; k++) o[k] = (k % 4 == 0) ? 1.0 : 0.0;
    } else {
      atomicAdd(bad + 1, 1);
    }
    return;
  }
  const double id = 1.0 / det;
  o[0] = c00 * id;
  o[1] = (a[2] * a[7] - a[1] * a[8]) * id;
  o[2] = (a[1] * a[5] - a[2] * a[4]) * id;
  o[3] = c01 * id;
  o[4] = (a[0] * a[8] - a[2] * a[6]) * id;
  o[5] = (a[2] * a[3] - a[0] * a[5]) * id;
  o[6] = c02 * id;
  o[7] = (a[1] * a[6] - a[0] * a[7]) * id;
  o[8] = (a[0] * a[4] - a[1] * a[3]) * id;
}

// y = A x with A = U + U^T - diag(U) from the upper blocks; four lanes per row
__global__ void __launch_bounds__(256) k_spmv(int N, const int *__restrict__ rows, const int *__restrict__ cols,
                                              const int *__restrict__ lrows, const int *__restrict__ lcols,
                                              const int *__restrict__ lslot, const double *__restrict__ vals,
                                              const double *__restrict__ x, double *__restrict__ y) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int r = (int)(t >> 2), sub = (int)(t & 3);
  double acc[3] = {0, 0, 0};
  if (r < N) {
    for (int s = rows[r] + sub; s < rows[r + 1]; s += 4) {
      const double *B = vals + 9 * (size_t)s;
      const double *xc = x + 3 * (size_t)cols[s];
      const double x0 = xc[0], x1 = xc[1], x2 = xc[2];
      acc[0] += B[0] * x0 + B[1] * x1 + B[2] * x2;
      acc[1] += B[3] * x0 + B[4] * x1 + B[5] * x2;
      acc[2] += B[6] * x0 + B[7] * x1 + B[8] * x2;
    }
    for (int q = lrows[r] + sub; q < lrows[r + 1]; q += 4) {
      const double *B = vals + 9 * (size_t)lslot[q];
      const double *xc = x + 3 * (size_t)lcols[q];
      const double x0 = xc[0], x1 = xc[1], x2 = xc[2];
      acc[0] += B[0] * x0 + B[3] * x1 + B[6] * x2;
      acc[1] += B[1] * x0 + B[4] * x1 + B[7] * x2;
      acc[2] += B[2] * x0 + B[5] * x1 + B[8] * x2;
    }
  }
#pragma unroll
  for (int o = 1; o <= 2; o <<= 1)
#pragma unroll
    for (int k = 0; k < 3; k++) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
  if (r < N && sub == 0) {
    y[3 * (size_t)r + 0] = acc[0];
    y[3 * (size_t)r + 1] = acc[1];
    y[3 * (size_t)r + 2] = acc[2];
  }
}

__device__ __forceinline__ double block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double s = 0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) s += sh[i];
  return s;
}

// ---- preconditioned MINRES (Paige & Saunders 1975), the matrix symmetric and
// possibly indefinite (softening cohesive zones), the preconditioner the SPD
// 3x3 block-Jacobi M.  Scalars live on the device:
//   sc[0] beta  [1] oldb  [2] alfa  [3] dbar  [4] epsln  [5] oldeps
//   sc[6] cs    [7] sn    [8] phibar [9] beta1 [10] phi   [11] delta
//   sc[12] gamma [13] breakdown flag
constexpr int NSC = 16;

// y = Dinv r for 3-vectors of N rows
__device__ __forceinline__ void apply_dinv(const double *D, const double r[3], double z[3]) {
#pragma unroll
  for (int k = 0; k < 3; k++) z[k] = D[3 * k] * r[0] + D[3 * k + 1] * r[1] + D[3 * k + 2] * r[2];
}

// start: x = 0, r1 = r2 = b, y = Dinv b, w = w2 = 0
__global__ void k_mr_start(int N, const double *__restrict__ b, const double *__restrict__ dinv,
                           double *__restrict__ x, double *__restrict__ r1, double *__restrict__ r2,
                           double *__restrict__ y, double *__restrict__ w, double *__restrict__ w2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double rv[3], z[3];
#pragma unroll
  for (int k = 0; k < 3; k++) rv[k] = b[3 * (size_t)i + k];
  apply_dinv(dinv + 9 * (size_t)i, rv, z);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const size_t j = 3 * (size_t)i + k;
    x[j] = 0;
    r1[j] = rv[k];
    r2[j] = rv[k];
    y[j] = z[k];
    w[j] = 0;
    w2[j] = 0;
  }
}

__global__ void k_mr_init(const double *__restrict__ part, double *__restrict__ sc) {
  if (threadIdx.x != 0) return;
  double b2 = 0;
  for (int i = 0; i < RED_BLOCKS; i++) b2 += part[i];
  for (int k = 0; k < NSC; k++) sc[k] = 0;
  if (b2 < 0 || !isfinite(b2)) sc[13] = 1;
  const double beta1 = b2 > 0 ? sqrt(b2) : 0.0;
  sc[0] = beta1;  // beta
  sc[1] = 0;      // oldb
  sc[6] = -1;     // cs
  sc[7] = 0;      // sn
  sc[8] = beta1;  // phibar
  sc[9] = beta1;  // beta1
}

// v = y / beta
__global__ void k_mr_v(int n, const double *__restrict__ sc, const double *__restrict__ y, double *__restrict__ v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  v[i] = sc[0] > 0 ? y[i] / sc[0] : 0.0;  // beta = 0: converged exactly, nothing left to add
}

// y -= (beta / oldb) r1 (after the first iteration); partial sums of v.y
__global__ void __launch_bounds__(256) k_mr_a(int n, int first, const double *__restrict__ sc,
                                              const double *__restrict__ r1, const double *__restrict__ v,
                                              double *__restrict__ y, double *__restrict__ part) {
  __shared__ double sh[8];
  const double f = (first || !(sc[1] > 0)) ? 0.0 : sc[0] / sc[1];
  double acc = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double yi = y[i] - f * r1[i];
    y[i] = yi;
    acc += v[i] * yi;
  }
  const double t = block_sum(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

__global__ void k_mr_alfa(const double *__restrict__ part, double *__restrict__ sc) {
  if (threadIdx.x != 0) return;
  double a = 0;
  for (int i = 0; i < RED_BLOCKS; i++) a += part[i];
  sc[2] = a;
}

// y -= (alfa / beta) r2; r1 = r2; r2 = y; y = Dinv r2; partial sums of r2.y
__global__ void __launch_bounds__(256) k_mr_b(int N, const double *__restrict__ sc, const double *__restrict__ dinv,
                                              double *__restrict__ r1, double *__restrict__ r2,
                                              double *__restrict__ y, double *__restrict__ part) {
  __shared__ double sh[8];
  const double f = sc[0] > 0 ? sc[2] / sc[0] : 0.0;
  double acc = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    double yv[3], z[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const size_t j = 3 * (size_t)i + k;
      yv[k] = y[j] - f * r2[j];
      r1[j] = r2[j];
      r2[j] = yv[k];
    }
    apply_dinv(dinv + 9 * (size_t)i, yv, z);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      y[3 * (size_t)i + k] = z[k];
      acc += yv[k] * z[k];
    }
  }
  const double t = block_sum(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// the plane rotation of this iteration
__global__ void k_mr_rot(const double *__restrict__ part, double *__restrict__ sc) {
  if (threadIdx.x != 0) return;
  double b2 = 0;
  for (int i = 0; i < RED_BLOCKS; i++) b2 += part[i];
  if (b2 < 0 || !isfinite(b2)) {
    sc[13] = 1;
    b2 = 0;
  }
  const double oldb = sc[0], beta = sqrt(b2), alfa = sc[2];
  const double cs = sc[6], sn = sc[7], dbar = sc[3];
  const double oldeps = sc[4];
  const double delta = cs * dbar + sn * alfa;
  const double gbar = sn * dbar - cs * alfa;
  const double epsln = sn * beta;
  const double dbar2 = -cs * beta;
  double gamma = sqrt(gbar * gbar + beta * beta);
  if (gamma < 1e-300) gamma = 1e-300;
  const double cs2 = gbar / gamma, sn2 = beta / gamma;
  const double phi = cs2 * sc[8];
  sc[8] = sn2 * sc[8];  // phibar
  sc[1] = oldb;
  sc[0] = beta;
  sc[3] = dbar2;
  sc[4] = epsln;
  sc[5] = oldeps;
  sc[6] = cs2;
  sc[7] = sn2;
  sc[10] = phi;
  sc[11] = delta;
  sc[12] = gamma;
}

// w1 = w2; w2 = w; w = (v - oldeps w1 - delta w2) / gamma; x += phi w
__global__ void k_mr_x(int n, const double *__restrict__ sc, const double *__restrict__ v, double *__restrict__ w,
                       double *__restrict__ w2, double *__restrict__ x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double w1 = w2[i], wo = w[i];
  const double wn = (v[i] - sc[5] * w1 - sc[11] * wo) / sc[12];
  w2[i] = wo;
  w[i] = wn;
  x[i] += sc[10] * wn;
}

// partial sums of b.y (the start's preconditioned norm)
__global__ void __launch_bounds__(256) k_dot(int n, const double *__restrict__ a, const double *__restrict__ b,
                                             double *__restrict__ part) {
  __shared__ double sh[8];
  double s1 = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s1 += a[i] * b[i];
  const double t = block_sum(s1, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

template <typename T>
int grow(icf_ctx *ctx, T **p, long long *cap, long long n) {
  if (n <= *cap && *p) return ICF_OK;
  cudaFree(*p);
  *p = nullptr;
  const long long c = n + n / 4 + 16;
  ICF_CUDA(ctx, cudaMalloc(p, sizeof(T) * (size_t)c));
  *cap = c;
  return ICF_OK;
}

}  // namespace

void icf_free_solver(icf_ctx *ctx) {
  icf_solver &S = ctx->solver;
  void *ptrs[] = {S.lrows, S.lcols, S.lslot, S.x, S.r, S.z, S.p, S.q, S.w, S.w2, S.dinv, S.part, S.sc};
  for (void *p : ptrs) cudaFree(p);
  if (S.h_sc) cudaFreeHost(S.h_sc);
  S = icf_solver();
}

// Lower-block index of the current structure (rebuilt when it changes).
static int build_lower(icf_ctx *ctx) {
  icf_solver &S = ctx->solver;
  cudaStream_t s = ctx->stream;
  const int N = ctx->N, nnz = ctx->nnz;
  ICF_TRY_RC(grow(ctx, &S.lrows, &S.rows_cap, N + 1));
  ICF_TRY_RC(grow(ctx, &S.lcols, &S.l_cap, nnz));
  ICF_TRY_RC(grow(ctx, &S.lslot, &S.ls_cap, nnz));
  unsigned long long *k0, *k1;
  int *s0;
  ICF_CUDA(ctx, cudaMallocAsync(&k0, sizeof(unsigned long long) * (size_t)nnz, s));
  ICF_CUDA(ctx, cudaMallocAsync(&k1, sizeof(unsigned long long) * (size_t)nnz, s));
  ICF_CUDA(ctx, cudaMallocAsync(&s0, sizeof(int) * (size_t)nnz, s));
  k_lower_keys<<<icf_blocks(nnz, 256), 256, 0, s>>>(nnz, ctx->d_mkeys, k0, s0);
  size_t tb = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, k0, k1, s0, S.lslot, nnz, 0, 64, s);
  if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
  ICF_CUDA(ctx, cub::DeviceRadixSort::SortPairs(ctx->d_tmp, tb, k0, k1, s0, S.lslot, nnz, 0, 64, s));
  k_lower_rows<<<icf_blocks(N + 1LL, 256), 256, 0, s>>>(N, nnz, k1, S.lrows, S.lcols);
  ICF_CUDA(ctx, cudaGetLastError());
  ICF_CUDA(ctx, cudaFreeAsync(k0, s));
  ICF_CUDA(ctx, cudaFreeAsync(k1, s));
  ICF_CUDA(ctx, cudaFreeAsync(s0, s));
  S.gen = ctx->struct_gen;
  return ICF_OK;
}

int icf_solve_impl(icf_ctx *ctx, double rel_tol, int max_iter, int *iters, double *relres) {
  icf_solver &S = ctx->solver;
  cudaStream_t s = ctx->stream;
  const int N = ctx->N;
  const long long n3 = 3LL * N;
  if (S.gen != ctx->struct_gen) ICF_TRY_RC(build_lower(ctx));
  // vectors: x, r1 (r), r2 (z), y (p), v (q), w, w2
  ICF_TRY_RC(grow(ctx, &S.x, &S.x_cap, n3));
  ICF_TRY_RC(grow(ctx, &S.r, &S.r_cap, n3));
  ICF_TRY_RC(grow(ctx, &S.z, &S.z_cap, n3));
  ICF_TRY_RC(grow(ctx, &S.p, &S.p_cap, n3));
  ICF_TRY_RC(grow(ctx, &S.q, &S.q_cap, n3));
  ICF_TRY_RC(grow(ctx, &S.w, &S.w_cap, n3));
  ICF_TRY_RC(grow(ctx, &S.w2, &S.w2_cap, n3));
  ICF_TRY_RC(grow(ctx, &S.dinv, &S.d_cap, 9LL * N));
  if (!S.part) ICF_CUDA(ctx, cudaMalloc(&S.part, sizeof(double) * 2 * RED_BLOCKS));
  if (!S.sc) ICF_CUDA(ctx, cudaMalloc(&S.sc, sizeof(double) * NSC + 2 * sizeof(int)));
  if (!S.h_sc) ICF_CUDA(ctx, cudaMallocHost(&S.h_sc, sizeof(double) * NSC));
  double *x = S.x, *r1 = S.r, *r2 = S.z, *y = S.p, *v = S.q;
  int *bad = reinterpret_cast<int *>(S.sc + NSC);
  ICF_CUDA(ctx, cudaMemsetAsync(bad, 0, 2 * sizeof(int), s));
  k_dinv<<<icf_blocks(N, 256), 256, 0, s>>>(N, ctx->d_rows, ctx->d_vals, S.dinv, bad);
  k_mr_start<<<icf_blocks(N, 256), 256, 0, s>>>(N, ctx->d_rhs, S.dinv, x, r1, r2, y, S.w, S.w2);
  k_dot<<<RED_BLOCKS, 256, 0, s>>>((int)n3, r1, y, S.part);
  k_mr_init<<<1, 32, 0, s>>>(S.part, S.sc);
  ICF_CUDA(ctx, cudaGetLastError());
  int it = 0;
  double rel = 0;
  const int check_every = 4;
  while (true) {
    ICF_CUDA(ctx, cudaMemcpyAsync(S.h_sc, S.sc, sizeof(double) * NSC, cudaMemcpyDeviceToHost, s));
    ICF_CUDA(ctx, cudaStreamSynchronize(s));
    const double phibar = S.h_sc[8], beta1 = S.h_sc[9];
    if (S.h_sc[13] != 0)
      return icf_fail(ctx, ICF_ERR_NUMERIC, "linear solve: breakdown (preconditioned residual norm negative or not finite)");
    rel = beta1 > 0 ? phibar / beta1 : 0.0;
    if (!std::isfinite(rel)) return icf_fail(ctx, ICF_ERR_NUMERIC, "linear solve: non-finite residual");
    if (rel <= rel_tol || beta1 == 0 || it >= max_iter) break;
    for (int k = 0; k < check_every && it < max_iter; k++, it++) {
      k_mr_v<<<icf_blocks(n3, 256), 256, 0, s>>>((int)n3, S.sc, y, v);
      k_spmv<<<icf_blocks(4LL * N, 256), 256, 0, s>>>(N, ctx->d_rows, ctx->d_cols, S.lrows, S.lcols, S.lslot,
                                                      ctx->d_vals, v, y);
      k_mr_a<<<RED_BLOCKS, 256, 0, s>>>((int)n3, it == 0 ? 1 : 0, S.sc, r1, v, y, S.part);
      k_mr_alfa<<<1, 32, 0, s>>>(S.part, S.sc);
      k_mr_b<<<RED_BLOCKS, 256, 0, s>>>(N, S.sc, S.dinv, r1, r2, y, S.part);
      k_mr_rot<<<1, 32, 0, s>>>(S.part, S.sc);
      k_mr_x<<<icf_blocks(n3, 256), 256, 0, s>>>((int)n3, S.sc, v, S.w, S.w2, x);
    }
    ICF_CUDA(ctx, cudaGetLastError());
  }
  int hbad[2] = {0, 0};
  ICF_CUDA(ctx, cudaMemcpy(hbad, bad, 2 * sizeof(int), cudaMemcpyDeviceToHost));
  if (hbad[0]) return icf_fail(ctx, ICF_ERR_NUMERIC, "linear solve: zero or non-finite diagonal block");
  S.n_indefinite = hbad[1];
  if (iters) *iters = it;
  if (relres) *relres = rel;
  if (rel > rel_tol && it >= max_iter)
  {
    char buf[64];
    snprintf(buf, sizeof(buf), "%.3e", rel);
    return icf_fail(ctx, ICF_ERR_NUMERIC, "linear solve: no convergence in " + std::to_string(max_iter) +
                                              " iterations (relative residual " + buf + ")");
  }
  return ICF_OK;
}
