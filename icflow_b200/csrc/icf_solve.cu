// icf_solve.cu -- the Newton linear solve on the device.
//
// The reference copies the upper-triangular BCSR matrix and the rhs to the
// host every Newton iteration and solves them with MKL PARDISO (symmetric,
// mtype -2, BSR 3x3; LinearSystem.cs:45-64, PardisoLoader2/dllmain.cpp:30-79).
// Here the system stays where it was assembled and is solved by conjugate
// gradients with a block-Jacobi (3x3) preconditioner:
//   - A x uses the stored upper blocks directly and their transposes through
//     a per-structure index of the lower blocks (row = column of the upper
//     block), four lanes per row and a fixed shuffle tree, so every product
//     is deterministic;
//   - dot products reduce per block and then in one block, in a fixed order;
//   - the CG scalars live on the device; the host reads the residual every
//     few iterations only to stop.
// The solution stays on the device for icf_apply_dx (du += dx, the
// reference's _XtoDU, ImplicitModel3.cs:247-256).
#include <cub/cub.cuh>

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

// inverse of each diagonal block (the first block of its row)
__global__ void k_dinv(int N, const int *__restrict__ rows, const double *__restrict__ vals,
                       double *__restrict__ dinv, int *__restrict__ bad) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= N) return;
  const double *a = vals + 9 * (size_t)rows[r];
  const double c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8], c02 = a[3] * a[7] - a[4] * a[6];
  const double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
  double *o = dinv + 9 * (size_t)r;
  if (!(fabs(det) > 0) || !isfinite(det)) {
    atomicOr(bad, 1);
    for (int k = 0; k < 9; k++) o[k] = (k % 4 == 0) ? 1.0 : 0.0;
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

// partial sums of a.b (and of c.d when c != nullptr) per block
__global__ void __launch_bounds__(256) k_dot2(int n, const double *__restrict__ a, const double *__restrict__ b,
                                              const double *__restrict__ c, const double *__restrict__ d,
                                              double *__restrict__ part) {
  __shared__ double sh[8];
  double s1 = 0, s2 = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    s1 += a[i] * b[i];
    if (c) s2 += c[i] * d[i];
  }
  const double t1 = block_sum(s1, sh);
  const double t2 = block_sum(s2, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = t1;
    part[RED_BLOCKS + blockIdx.x] = t2;
  }
}

// scalars: [0] rz  [1] alpha  [2] beta  [3] rr  [4] bb  [5] breakdown
__global__ void k_alpha(const double *__restrict__ part, double *__restrict__ sc) {
  if (threadIdx.x != 0) return;
  double pq = 0;
  for (int i = 0; i < RED_BLOCKS; i++) pq += part[i];
  if (!(pq > 0) || !isfinite(pq)) {
    sc[1] = 0;
    sc[5] = 1;
  } else {
    sc[1] = sc[0] / pq;
  }
}
__global__ void k_beta(const double *__restrict__ part, double *__restrict__ sc, int init) {
  if (threadIdx.x != 0) return;
  double rz = 0, rr = 0;
  for (int i = 0; i < RED_BLOCKS; i++) rz += part[i];
  for (int i = 0; i < RED_BLOCKS; i++) rr += part[RED_BLOCKS + i];
  if (init) {
    sc[4] = rr;
    sc[5] = 0;
    sc[2] = 0;
  } else {
    sc[2] = sc[0] > 0 ? rz / sc[0] : 0;
  }
  sc[0] = rz;
  sc[3] = rr;
}

// x += alpha p; r -= alpha q; z = Dinv r
__global__ void k_update(int N, const double *__restrict__ sc, const double *__restrict__ p,
                         const double *__restrict__ q, const double *__restrict__ dinv, double *__restrict__ x,
                         double *__restrict__ r, double *__restrict__ z) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double al = sc[1];
  double rv[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const size_t j = 3 * (size_t)i + k;
    x[j] += al * p[j];
    rv[k] = r[j] - al * q[j];
    r[j] = rv[k];
  }
  const double *D = dinv + 9 * (size_t)i;
#pragma unroll
  for (int k = 0; k < 3; k++) z[3 * (size_t)i + k] = D[3 * k] * rv[0] + D[3 * k + 1] * rv[1] + D[3 * k + 2] * rv[2];
}

// start: x = 0, r = b, z = Dinv r
__global__ void k_start(int N, const double *__restrict__ b, const double *__restrict__ dinv, double *__restrict__ x,
                        double *__restrict__ r, double *__restrict__ z, double *__restrict__ p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double rv[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const size_t j = 3 * (size_t)i + k;
    x[j] = 0;
    rv[k] = b[j];
    r[j] = rv[k];
  }
  const double *D = dinv + 9 * (size_t)i;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const double zk = D[3 * k] * rv[0] + D[3 * k + 1] * rv[1] + D[3 * k + 2] * rv[2];
    z[3 * (size_t)i + k] = zk;
    p[3 * (size_t)i + k] = zk;
  }
}

__global__ void k_newp(int n, const double *__restrict__ sc, const double *__restrict__ z, double *__restrict__ p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  p[i] = z[i] + sc[2] * p[i];
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
  void *ptrs[] = {S.lrows, S.lcols, S.lslot, S.x, S.r, S.z, S.p, S.q, S.dinv, S.part, S.sc};
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
  ICF_TRY_RC(grow(ctx, &S.x, &S.x_cap, n3));
  ICF_TRY_RC(grow(ctx, &S.r, &S.r_cap, n3));
  ICF_TRY_RC(grow(ctx, &S.z, &S.z_cap, n3));
  ICF_TRY_RC(grow(ctx, &S.p, &S.p_cap, n3));
  ICF_TRY_RC(grow(ctx, &S.q, &S.q_cap, n3));
  ICF_TRY_RC(grow(ctx, &S.dinv, &S.d_cap, 9LL * N));
  if (!S.part) ICF_CUDA(ctx, cudaMalloc(&S.part, sizeof(double) * 2 * RED_BLOCKS));
  if (!S.sc) ICF_CUDA(ctx, cudaMalloc(&S.sc, sizeof(double) * 8 + sizeof(int)));
  if (!S.h_sc) ICF_CUDA(ctx, cudaMallocHost(&S.h_sc, sizeof(double) * 8));
  int *bad = reinterpret_cast<int *>(S.sc + 8);
  ICF_CUDA(ctx, cudaMemsetAsync(bad, 0, sizeof(int), s));
  k_dinv<<<icf_blocks(N, 256), 256, 0, s>>>(N, ctx->d_rows, ctx->d_vals, S.dinv, bad);
  k_start<<<icf_blocks(N, 256), 256, 0, s>>>(N, ctx->d_rhs, S.dinv, S.x, S.r, S.z, S.p);
  k_dot2<<<RED_BLOCKS, 256, 0, s>>>((int)n3, S.r, S.z, S.r, S.r, S.part);
  k_beta<<<1, 32, 0, s>>>(S.part, S.sc, 1);
  ICF_CUDA(ctx, cudaGetLastError());
  int it = 0;
  double rel = 0;
  const int check_every = 4;
  bool done = false;
  while (!done) {
    ICF_CUDA(ctx, cudaMemcpyAsync(S.h_sc, S.sc, sizeof(double) * 8, cudaMemcpyDeviceToHost, s));
    ICF_CUDA(ctx, cudaStreamSynchronize(s));
    const double rr = S.h_sc[3], bb = S.h_sc[4];
    rel = bb > 0 ? std::sqrt(rr / bb) : 0.0;
    if (!std::isfinite(rel)) return icf_fail(ctx, ICF_ERR_NUMERIC, "linear solve: non-finite residual");
    if (S.h_sc[5] != 0) return icf_fail(ctx, ICF_ERR_NUMERIC, "linear solve: CG breakdown (matrix not positive definite)");
    if (rel <= rel_tol || bb == 0) break;
    if (it >= max_iter) break;
    for (int k = 0; k < check_every && it < max_iter; k++, it++) {
      k_spmv<<<icf_blocks(4LL * N, 256), 256, 0, s>>>(N, ctx->d_rows, ctx->d_cols, S.lrows, S.lcols, S.lslot,
                                                      ctx->d_vals, S.p, S.q);
      k_dot2<<<RED_BLOCKS, 256, 0, s>>>((int)n3, S.p, S.q, nullptr, nullptr, S.part);
      k_alpha<<<1, 32, 0, s>>>(S.part, S.sc);
      k_update<<<icf_blocks(N, 256), 256, 0, s>>>(N, S.sc, S.p, S.q, S.dinv, S.x, S.r, S.z);
      k_dot2<<<RED_BLOCKS, 256, 0, s>>>((int)n3, S.r, S.z, S.r, S.r, S.part);
      k_beta<<<1, 32, 0, s>>>(S.part, S.sc, 0);
      k_newp<<<icf_blocks(n3, 256), 256, 0, s>>>((int)n3, S.sc, S.z, S.p);
    }
    ICF_CUDA(ctx, cudaGetLastError());
  }
  int hbad = 0;
  ICF_CUDA(ctx, cudaMemcpy(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost));
  if (hbad) return icf_fail(ctx, ICF_ERR_NUMERIC, "linear solve: singular diagonal block");
  if (iters) *iters = it;
  if (relres) *relres = rel;
  if (rel > rel_tol && it >= max_iter)
    return icf_fail(ctx, ICF_ERR_NUMERIC, "linear solve: no convergence in " + std::to_string(max_iter) +
                                              " iterations (relative residual " + std::to_string(rel) + ")");
  return ICF_OK;
}
