// icf_mlp.cu -- the learned Newton warm start: a per-node MLP 15 -> 64 -> 64 -> 3
// with GELU, BF16 weights and FP32 accumulation, with its own training.
//
// No counterpart in the reference: icFlow starts every Newton loop from
// du = v h (ImplicitModel3.cs:149-156).  The network predicts a correction
// to that guess from each node's (u, v, a, du_{n-1}, du_{n-2}) (15 inputs,
// normalised with fixed per-input shifts and scales); the guess is
// du = v h + out_scale * net(x).  With a zero network the plain guess comes
// back unchanged.
//
// Forward: one warp per 16 nodes, bf16 mma.sync m16n8k16 with FP32
// accumulators; each layer's accumulator fragments are re-used in registers
// as the next layer's A fragments (the C layout of two adjacent 8-column
// tiles is the A layout of one 16-column k-step).  Weights sit in shared
// memory as bf16.  Rounding points: the inputs and the two hidden activations
// are rounded to bf16 before each product; biases, GELU and all sums are
// FP32.
//
// Training: the forward above (keeping Z1, H1, Z2, H2), then the backward in
// FP32 CUDA-core arithmetic, per-chunk weight-gradient partials and a fixed
// order reduction (no atomics: a gradient is identical run to run), and Adam
// on FP32 master weights, after which the bf16 copies are refreshed.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <utility>
#include <cstring>
#include <string>
#include <vector>

#include "icf_internal.cuh"

#define NI 15   // inputs
#define NH 64   // hidden width
#define NO 3    // outputs
// parameter layout: W1[64][15] b1[64] W2[64][64] b2[64] W3[3][64] b3[3]
#define OFF_W1 0
#define OFF_B1 (OFF_W1 + NH * NI)
#define OFF_W2 (OFF_B1 + NH)
#define OFF_B2 (OFF_W2 + NH * NH)
#define OFF_W3 (OFF_B2 + NH)
#define OFF_B3 (OFF_W3 + NO * NH)
#define NPAR (OFF_B3 + NO)

struct icf_mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  float *d_master = nullptr;  // FP32 parameters (NPAR)
  float *d_m = nullptr, *d_v = nullptr;  // Adam moments
  __nv_bfloat16 *d_wb = nullptr;  // bf16 weights, padded: W1 64x16, W2 64x64, W3 8x64
  float *d_norm = nullptr;        // in_shift[15], in_scale[15], out_scale[3]
  long long adam_t = 0;
  // training buffers
  int cap = 0;
  float *d_x = nullptr, *d_y = nullptr;
  float *d_z1 = nullptr, *d_h1 = nullptr, *d_z2 = nullptr, *d_h2 = nullptr, *d_out = nullptr;
  float *d_dy = nullptr, *d_dz1 = nullptr, *d_dz2 = nullptr;
  float *d_part = nullptr;  // per-chunk gradient partials
  int part_cap = 0;
  float *d_grad = nullptr, *d_loss = nullptr;
};

namespace {

constexpr int WB_W1 = 0, WB_W2 = NH * 16, WB_W3 = WB_W2 + NH * NH, WB_N = WB_W3 + 8 * NH;

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
// d/dz GELU = Phi(z) + z phi(z)
__device__ __forceinline__ float gelu_d(float z) {
  const float Phi = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
  const float phi = 0.39894228040143268f * expf(-0.5f * z * z);
  return Phi + z * phi;
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&v);
}
__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// B fragment of W (row-major [rows][ld] bf16) for n-tile j, k-step kk:
// element (k, n) = W[8j + n][16kk + k]
__device__ __forceinline__ void bfrag(const __nv_bfloat16 *W, int ld, int j, int kk, int lane, uint32_t b[2]) {
  const int g = lane >> 2, t = lane & 3;
  const __nv_bfloat16 *row = W + (size_t)(8 * j + g) * ld + 16 * kk + 2 * t;
  b[0] = *reinterpret_cast<const uint32_t *>(row);
  b[1] = *reinterpret_cast<const uint32_t *>(row + 8);
}

struct fwd_out {
  float z1[8][4], z2[8][4], y[4];
};

// Forward of 16 nodes [r0, r0 + 16) (rows >= n read as zeros).  Inputs are
// normalised here.  Returns the pre-activations and the output fragment.
__device__ __forceinline__ void mlp_forward16(const float *__restrict__ x, int n, int r0, const __nv_bfloat16 *sW,
                                              const float *sB, const float *sNorm, int lane, fwd_out &f) {
  const int g = lane >> 2, t = lane & 3;
  // A fragment of the normalised inputs (16 x 16, column 15 zero)
  auto xin = [&](int r, int c) -> float {
    if (r >= n || c >= NI) return 0.f;
    return (x[(size_t)r * NI + c] - sNorm[c]) * sNorm[NI + c];
  };
  uint32_t a[4];
  a[0] = pack_bf16(xin(r0 + g, 2 * t), xin(r0 + g, 2 * t + 1));
  a[1] = pack_bf16(xin(r0 + g + 8, 2 * t), xin(r0 + g + 8, 2 * t + 1));
  a[2] = pack_bf16(xin(r0 + g, 2 * t + 8), xin(r0 + g, 2 * t + 9));
  a[3] = pack_bf16(xin(r0 + g + 8, 2 * t + 8), xin(r0 + g + 8, 2 * t + 9));
  // layer 1
#pragma unroll
  for (int j = 0; j < 8; j++) {
    f.z1[j][0] = f.z1[j][1] = f.z1[j][2] = f.z1[j][3] = 0.f;
    uint32_t b[2];
    bfrag(sW + WB_W1, 16, j, 0, lane, b);
    mma_bf16(f.z1[j], a, b);
    const float b0 = sB[OFF_B1 + 8 * j + 2 * t], b1 = sB[OFF_B1 + 8 * j + 2 * t + 1];
    f.z1[j][0] += b0; f.z1[j][1] += b1; f.z1[j][2] += b0; f.z1[j][3] += b1;
  }
  // layer 2: A fragments from GELU(z1) of tiles 2kk, 2kk + 1
#pragma unroll
  for (int j = 0; j < 8; j++) f.z2[j][0] = f.z2[j][1] = f.z2[j][2] = f.z2[j][3] = 0.f;
#pragma unroll
  for (int kk = 0; kk < 4; kk++) {
    uint32_t ah[4];
    ah[0] = pack_bf16(gelu(f.z1[2 * kk][0]), gelu(f.z1[2 * kk][1]));
    ah[1] = pack_bf16(gelu(f.z1[2 * kk][2]), gelu(f.z1[2 * kk][3]));
    ah[2] = pack_bf16(gelu(f.z1[2 * kk + 1][0]), gelu(f.z1[2 * kk + 1][1]));
    ah[3] = pack_bf16(gelu(f.z1[2 * kk + 1][2]), gelu(f.z1[2 * kk + 1][3]));
#pragma unroll
    for (int j = 0; j < 8; j++) {
      uint32_t b[2];
      bfrag(sW + WB_W2, NH, j, kk, lane, b);
      mma_bf16(f.z2[j], ah, b);
    }
  }
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const float b0 = sB[OFF_B2 + 8 * j + 2 * t], b1 = sB[OFF_B2 + 8 * j + 2 * t + 1];
    f.z2[j][0] += b0; f.z2[j][1] += b1; f.z2[j][2] += b0; f.z2[j][3] += b1;
  }
  // layer 3 (W3 padded to 8 rows)
  f.y[0] = f.y[1] = f.y[2] = f.y[3] = 0.f;
#pragma unroll
  for (int kk = 0; kk < 4; kk++) {
    uint32_t ah[4];
    ah[0] = pack_bf16(gelu(f.z2[2 * kk][0]), gelu(f.z2[2 * kk][1]));
    ah[1] = pack_bf16(gelu(f.z2[2 * kk][2]), gelu(f.z2[2 * kk][3]));
    ah[2] = pack_bf16(gelu(f.z2[2 * kk + 1][0]), gelu(f.z2[2 * kk + 1][1]));
    ah[3] = pack_bf16(gelu(f.z2[2 * kk + 1][2]), gelu(f.z2[2 * kk + 1][3]));
    uint32_t b[2];
    bfrag(sW + WB_W3, NH, 0, kk, lane, b);
    mma_bf16(f.y, ah, b);
  }
  const int c0 = 2 * t, c1 = 2 * t + 1;
  if (c0 < NO) { f.y[0] += sB[OFF_B3 + c0]; f.y[2] += sB[OFF_B3 + c0]; }
  if (c1 < NO) { f.y[1] += sB[OFF_B3 + c1]; f.y[3] += sB[OFF_B3 + c1]; }
}

__device__ __forceinline__ void load_params(const __nv_bfloat16 *wb, const float *master, const float *norm,
                                            __nv_bfloat16 *sW, float *sB, float *sNorm) {
  for (int i = threadIdx.x; i < WB_N; i += blockDim.x) sW[i] = wb[i];
  for (int i = threadIdx.x; i < NPAR; i += blockDim.x) sB[i] = master[i];
  for (int i = threadIdx.x; i < 2 * NI + NO; i += blockDim.x) sNorm[i] = norm[i];
  __syncthreads();
}

// inference: y[n][3] = network output (normalised output units)
__global__ void __launch_bounds__(256) k_mlp_infer(int n, const float *__restrict__ x, const __nv_bfloat16 *wb,
                                                   const float *master, const float *norm, float *__restrict__ y) {
  __shared__ __nv_bfloat16 sW[WB_N];
  __shared__ float sB[NPAR];
  __shared__ float sNorm[2 * NI + NO];
  load_params(wb, master, norm, sW, sB, sNorm);
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int r0 = 16 * warp; r0 < n; r0 += 16 * nwarps) {
    fwd_out f;
    mlp_forward16(x, n, r0, sW, sB, sNorm, lane, f);
    const int g = lane >> 2, t = lane & 3;
    const int c0 = 2 * t, c1 = 2 * t + 1;
    if (r0 + g < n) {
      if (c0 < NO) y[(size_t)(r0 + g) * NO + c0] = f.y[0];
      if (c1 < NO) y[(size_t)(r0 + g) * NO + c1] = f.y[1];
    }
    if (r0 + g + 8 < n) {
      if (c0 < NO) y[(size_t)(r0 + g + 8) * NO + c0] = f.y[2];
      if (c1 < NO) y[(size_t)(r0 + g + 8) * NO + c1] = f.y[3];
    }
  }
}

// training forward: keeps Z1, H1 = bf16(GELU(Z1)), Z2, H2 and dY = 2 (y - t) / n
// (mean squared error over nodes and components); loss partial per warp-tile
__global__ void __launch_bounds__(256) k_mlp_fwd_train(int n, const float *__restrict__ x, const float *__restrict__ tgt,
                                                       const __nv_bfloat16 *wb, const float *master,
                                                       const float *norm, float *__restrict__ z1,
                                                       float *__restrict__ h1, float *__restrict__ z2,
                                                       float *__restrict__ h2, float *__restrict__ dy,
                                                       float *__restrict__ loss_part) {
  __shared__ __nv_bfloat16 sW[WB_N];
  __shared__ float sB[NPAR];
  __shared__ float sNorm[2 * NI + NO];
  load_params(wb, master, norm, sW, sB, sNorm);
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int r0 = 16 * warp;
  float l = 0.f;
  if (r0 < n) {
    fwd_out f;
    mlp_forward16(x, n, r0, sW, sB, sNorm, lane, f);
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int j = 0; j < 8; j++)
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int r = r0 + g + (e >= 2 ? 8 : 0), c = 8 * j + 2 * t + (e & 1);
        if (r < n) {
          z1[(size_t)r * NH + c] = f.z1[j][e];
          h1[(size_t)r * NH + c] = bf16r(gelu(f.z1[j][e]));
          z2[(size_t)r * NH + c] = f.z2[j][e];
          h2[(size_t)r * NH + c] = bf16r(gelu(f.z2[j][e]));
        }
      }
    const float inv = 2.0f / (float)(n * NO);
    if (tgt != nullptr) {  // tgt == nullptr: dy was supplied by the caller
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int r = r0 + g + (e >= 2 ? 8 : 0), c = 2 * t + (e & 1);
        if (r < n && c < NO) {
          const float d = f.y[e] - tgt[(size_t)r * NO + c];
          dy[(size_t)r * NO + c] = inv * d;
          l += d * d;
        }
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
  if (lane == 0) loss_part[warp] = l;
}

// backward through the activations, one thread per node:
// dZ2 = (dY W3) * gelu'(Z2);  dZ1 = (dZ2 W2) * gelu'(Z1)   (W = bf16 values)
__global__ void __launch_bounds__(128) k_mlp_bwd_act(int n, const __nv_bfloat16 *wb, const float *__restrict__ z1,
                                                     const float *__restrict__ z2, const float *__restrict__ dy,
                                                     float *__restrict__ dz1, float *__restrict__ dz2) {
  __shared__ float sW2[NH * NH];
  __shared__ float sW3[NO * NH];
  for (int i = threadIdx.x; i < NH * NH; i += blockDim.x) sW2[i] = __bfloat162float(wb[WB_W2 + i]);
  for (int i = threadIdx.x; i < NO * NH; i += blockDim.x) sW3[i] = __bfloat162float(wb[WB_W3 + i]);
  __syncthreads();
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const float d0 = dy[(size_t)r * NO], d1 = dy[(size_t)r * NO + 1], d2 = dy[(size_t)r * NO + 2];
  float g2[NH];
#pragma unroll 8
  for (int j = 0; j < NH; j++) {
    const float dh = d0 * sW3[j] + d1 * sW3[NH + j] + d2 * sW3[2 * NH + j];
    g2[j] = dh * gelu_d(z2[(size_t)r * NH + j]);
    dz2[(size_t)r * NH + j] = g2[j];
  }
  for (int i = 0; i < NH; i++) {
    float dh = 0.f;
#pragma unroll 8
    for (int j = 0; j < NH; j++) dh += g2[j] * sW2[j * NH + i];
    dz1[(size_t)r * NH + i] = dh * gelu_d(z1[(size_t)r * NH + i]);
  }
}

constexpr int CHUNK = 1024;  // nodes per weight-gradient partial

// Partials of every weight and bias gradient over one chunk of nodes:
//   dW1 = dZ1^T Xn, db1 = sum dZ1, dW2 = dZ2^T H1, db2 = sum dZ2,
//   dW3 = dY^T H2, db3 = sum dY
// (Xn the bf16-rounded normalised inputs).  256 threads; thread i owns
// parameters i, i + 256, ... and walks the chunk in order.
__global__ void __launch_bounds__(256) k_mlp_wgrad(int n, const float *__restrict__ x, const float *norm,
                                                   const float *__restrict__ h1, const float *__restrict__ h2,
                                                   const float *__restrict__ dz1, const float *__restrict__ dz2,
                                                   const float *__restrict__ dy, float *__restrict__ part) {
  __shared__ float sx[32][NI], sh1[32][NH], sh2[32][NH], sg1[32][NH], sg2[32][NH], sdy[32][NO];
  constexpr int PER = (NPAR + 255) / 256;
  float acc[PER];
#pragma unroll
  for (int q = 0; q < PER; q++) acc[q] = 0.f;
  const int b0 = blockIdx.x * CHUNK, b1 = min(n, b0 + CHUNK);
  for (int s0 = b0; s0 < b1; s0 += 32) {
    const int m = min(32, b1 - s0);
    __syncthreads();
    for (int i = threadIdx.x; i < 32 * NH; i += blockDim.x) {
      const int r = i / NH, c = i % NH;
      const bool ok = r < m;
      sh1[r][c] = ok ? h1[(size_t)(s0 + r) * NH + c] : 0.f;
      sh2[r][c] = ok ? h2[(size_t)(s0 + r) * NH + c] : 0.f;
      sg1[r][c] = ok ? dz1[(size_t)(s0 + r) * NH + c] : 0.f;
      sg2[r][c] = ok ? dz2[(size_t)(s0 + r) * NH + c] : 0.f;
    }
    for (int i = threadIdx.x; i < 32 * NI; i += blockDim.x) {
      const int r = i / NI, c = i % NI;
      sx[r][c] = r < m ? bf16r((x[(size_t)(s0 + r) * NI + c] - norm[c]) * norm[NI + c]) : 0.f;
    }
    for (int i = threadIdx.x; i < 32 * NO; i += blockDim.x) {
      const int r = i / NO, c = i % NO;
      sdy[r][c] = r < m ? dy[(size_t)(s0 + r) * NO + c] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < PER; q++) {
      const int p = threadIdx.x + 256 * q;
      if (p >= NPAR) break;
      float s = 0.f;
      if (p < OFF_B1) {
        const int o = p / NI, i = p % NI;
        for (int r = 0; r < 32; r++) s += sg1[r][o] * sx[r][i];
      } else if (p < OFF_W2) {
        const int o = p - OFF_B1;
        for (int r = 0; r < 32; r++) s += sg1[r][o];
      } else if (p < OFF_B2) {
        const int o = (p - OFF_W2) / NH, i = (p - OFF_W2) % NH;
        for (int r = 0; r < 32; r++) s += sg2[r][o] * sh1[r][i];
      } else if (p < OFF_W3) {
        const int o = p - OFF_B2;
        for (int r = 0; r < 32; r++) s += sg2[r][o];
      } else if (p < OFF_B3) {
        const int o = (p - OFF_W3) / NH, i = (p - OFF_W3) % NH;
        for (int r = 0; r < 32; r++) s += sdy[r][o] * sh2[r][i];
      } else {
        const int o = p - OFF_B3;
        for (int r = 0; r < 32; r++) s += sdy[r][o];
      }
      acc[q] += s;
    }
  }
#pragma unroll
  for (int q = 0; q < PER; q++) {
    const int p = threadIdx.x + 256 * q;
    if (p < NPAR) part[(size_t)blockIdx.x * NPAR + p] = acc[q];
  }
}

// grad[p] = sum over chunks in order; loss = sum of warp partials / (n NO)
__global__ void k_mlp_reduce(int nchunks, const float *__restrict__ part, float *__restrict__ grad, int nloss,
                             const float *__restrict__ loss_part, float *loss, int n) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < NPAR) {
    float s = 0.f;
    for (int c = 0; c < nchunks; c++) s += part[(size_t)c * NPAR + p];
    grad[p] = s;
  }
  if (p == 0 && loss) {
    float l = 0.f;
    for (int i = 0; i < nloss; i++) l += loss_part[i];
    *loss = l / (float)(n * NO);
  }
}

// bf16 copies of the weights in the padded layout the forward reads
__global__ void k_mlp_pack(const float *__restrict__ master, __nv_bfloat16 *__restrict__ wb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= WB_N) return;
  float v = 0.f;
  if (i < WB_W2) {
    const int o = i / 16, k = i % 16;
    v = k < NI ? master[OFF_W1 + o * NI + k] : 0.f;
  } else if (i < WB_W3) {
    v = master[OFF_W2 + (i - WB_W2)];
  } else {
    const int o = (i - WB_W3) / NH, k = (i - WB_W3) % NH;
    v = o < NO ? master[OFF_W3 + o * NH + k] : 0.f;
  }
  wb[i] = __float2bfloat16_rn(v);
}

__global__ void k_mlp_adam(float *__restrict__ w, float *__restrict__ m, float *__restrict__ v,
                           const float *__restrict__ g, float lr, float b1c, float b2c) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= NPAR) return;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  m[p] = b1 * m[p] + (1.f - b1) * g[p];
  v[p] = b2 * v[p] + (1.f - b2) * g[p] * g[p];
  const float mh = m[p] / b1c, vh = v[p] / b2c;
  w[p] -= lr * mh / (sqrtf(vh) + eps);
}

__global__ void k_gather_rows(int k, const int *__restrict__ idx, const float *__restrict__ xa,
                              const float *__restrict__ ya, float *__restrict__ x, float *__restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= k) return;
  const int r = idx[i];
  for (int c = 0; c < NI; c++) x[(size_t)i * NI + c] = xa[(size_t)r * NI + c];
  for (int c = 0; c < NO; c++) y[(size_t)i * NO + c] = ya[(size_t)r * NO + c];
}

int fail(icf_mlp *m, int code, const std::string &msg) {
  m->err = msg;
  return code;
}
#define MLP_CUDA(m, call)                                                                          \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) return fail((m), ICF_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

int ensure_cap(icf_mlp *m, int n) {
  if (n <= m->cap) return ICF_OK;
  float **bufs[] = {&m->d_x, &m->d_y, &m->d_z1, &m->d_h1, &m->d_z2, &m->d_h2, &m->d_out, &m->d_dy, &m->d_dz1, &m->d_dz2};
  const size_t w[] = {NI, NO, NH, NH, NH, NH, NO, NO, NH, NH};
  for (int i = 0; i < 10; i++) {
    cudaFree(*bufs[i]);
    *bufs[i] = nullptr;
  }
  for (int i = 0; i < 10; i++) MLP_CUDA(m, cudaMalloc(bufs[i], sizeof(float) * w[i] * (size_t)n));
  m->cap = n;
  const int nch = (n + CHUNK - 1) / CHUNK;
  if (nch > m->part_cap) {
    cudaFree(m->d_part);
    m->d_part = nullptr;
    MLP_CUDA(m, cudaMalloc(&m->d_part, sizeof(float) * NPAR * (size_t)nch));
    m->part_cap = nch;
  }
  cudaFree(m->d_loss);
  m->d_loss = nullptr;
  MLP_CUDA(m, cudaMalloc(&m->d_loss, sizeof(float) * ((size_t)(n + 15) / 16 + 16)));
  return ICF_OK;
}

// forward + backward of the data already in d_x, d_y (n nodes): d_grad, loss.
// dy_given: d_dy already holds dL/dy (the caller's loss), d_y is unused.
int grad_on_device(icf_mlp *m, int n, float *loss_host, bool dy_given = false) {
  cudaStream_t s = m->stream;
  const int tiles = (n + 15) / 16;
  const int blocks = (tiles + 7) / 8;
  float *loss_part = m->d_loss + 1;
  k_mlp_fwd_train<<<blocks, 256, 0, s>>>(n, m->d_x, dy_given ? nullptr : m->d_y, m->d_wb, m->d_master, m->d_norm,
                                          m->d_z1, m->d_h1, m->d_z2, m->d_h2, m->d_dy, loss_part);
  // warps beyond the last tile wrote zero partials: count them in
  k_mlp_bwd_act<<<icf_blocks(n, 128), 128, 0, s>>>(n, m->d_wb, m->d_z1, m->d_z2, m->d_dy, m->d_dz1, m->d_dz2);
  const int nch = (n + CHUNK - 1) / CHUNK;
  k_mlp_wgrad<<<nch, 256, 0, s>>>(n, m->d_x, m->d_norm, m->d_h1, m->d_h2, m->d_dz1, m->d_dz2, m->d_dy, m->d_part);
  k_mlp_reduce<<<icf_blocks(NPAR, 256), 256, 0, s>>>(nch, m->d_part, m->d_grad, blocks * 8, loss_part, m->d_loss, n);
  MLP_CUDA(m, cudaGetLastError());
  if (loss_host) {
    MLP_CUDA(m, cudaMemcpyAsync(loss_host, m->d_loss, sizeof(float), cudaMemcpyDeviceToHost, s));
    MLP_CUDA(m, cudaStreamSynchronize(s));
  }
  return ICF_OK;
}

}  // namespace

extern "C" {

int icf_mlp_create(int device, icf_mlp **out) {
  if (!out) return ICF_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return ICF_ERR_NODEVICE;
  if (device < 0 || device >= ndev) return ICF_ERR_ARG;
  icf_mlp *m = new icf_mlp();
  m->device = device;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) ||
      cudaMalloc(&m->d_master, sizeof(float) * NPAR) || cudaMalloc(&m->d_m, sizeof(float) * NPAR) ||
      cudaMalloc(&m->d_v, sizeof(float) * NPAR) || cudaMalloc(&m->d_grad, sizeof(float) * NPAR) ||
      cudaMalloc(&m->d_wb, sizeof(__nv_bfloat16) * WB_N) || cudaMalloc(&m->d_norm, sizeof(float) * (2 * NI + NO))) {
    delete m;
    return ICF_ERR_CUDA;
  }
  std::vector<float> norm(2 * NI + NO, 0.f);
  for (int i = 0; i < NI; i++) norm[NI + i] = 1.f;
  for (int i = 0; i < NO; i++) norm[2 * NI + i] = 1.f;
  cudaMemcpy(m->d_norm, norm.data(), sizeof(float) * norm.size(), cudaMemcpyHostToDevice);
  cudaMemset(m->d_master, 0, sizeof(float) * NPAR);
  cudaMemset(m->d_m, 0, sizeof(float) * NPAR);
  cudaMemset(m->d_v, 0, sizeof(float) * NPAR);
  k_mlp_pack<<<icf_blocks(WB_N, 256), 256, 0, m->stream>>>(m->d_master, m->d_wb);
  if (cudaStreamSynchronize(m->stream) != cudaSuccess) {
    delete m;
    return ICF_ERR_CUDA;
  }
  *out = m;
  return ICF_OK;
}

int icf_mlp_destroy(icf_mlp *m) {
  if (!m) return ICF_ERR_ARG;
  cudaSetDevice(m->device);
  void *p[] = {m->d_master, m->d_m, m->d_v, m->d_wb, m->d_norm, m->d_x, m->d_y, m->d_z1, m->d_h1, m->d_z2,
               m->d_h2, m->d_out, m->d_dy, m->d_dz1, m->d_dz2, m->d_part, m->d_grad, m->d_loss};
  for (void *q : p) cudaFree(q);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
  return ICF_OK;
}

const char *icf_mlp_last_error(const icf_mlp *m) { return m ? m->err.c_str() : "null network"; }
int icf_mlp_param_count(void) { return NPAR; }

int icf_mlp_set_params(icf_mlp *m, const float *params, const float *norm) {
  if (!m || !params) return ICF_ERR_ARG;
  MLP_CUDA(m, cudaSetDevice(m->device));
  MLP_CUDA(m, cudaMemcpy(m->d_master, params, sizeof(float) * NPAR, cudaMemcpyHostToDevice));
  if (norm) MLP_CUDA(m, cudaMemcpy(m->d_norm, norm, sizeof(float) * (2 * NI + NO), cudaMemcpyHostToDevice));
  MLP_CUDA(m, cudaMemset(m->d_m, 0, sizeof(float) * NPAR));
  MLP_CUDA(m, cudaMemset(m->d_v, 0, sizeof(float) * NPAR));
  m->adam_t = 0;
  k_mlp_pack<<<icf_blocks(WB_N, 256), 256, 0, m->stream>>>(m->d_master, m->d_wb);
  MLP_CUDA(m, cudaStreamSynchronize(m->stream));
  return ICF_OK;
}

int icf_mlp_get_params(icf_mlp *m, float *params, float *norm) {
  if (!m || !params) return ICF_ERR_ARG;
  MLP_CUDA(m, cudaSetDevice(m->device));
  MLP_CUDA(m, cudaStreamSynchronize(m->stream));
  MLP_CUDA(m, cudaMemcpy(params, m->d_master, sizeof(float) * NPAR, cudaMemcpyDeviceToHost));
  if (norm) MLP_CUDA(m, cudaMemcpy(norm, m->d_norm, sizeof(float) * (2 * NI + NO), cudaMemcpyDeviceToHost));
  return ICF_OK;
}

int icf_mlp_forward(icf_mlp *m, int n, const float *x, float *y) {
  if (!m || n < 0 || (n && (!x || !y))) return ICF_ERR_ARG;
  if (n == 0) return ICF_OK;
  MLP_CUDA(m, cudaSetDevice(m->device));
  if (ensure_cap(m, n)) return ICF_ERR_CUDA;
  cudaStream_t s = m->stream;
  MLP_CUDA(m, cudaMemcpyAsync(m->d_x, x, sizeof(float) * NI * (size_t)n, cudaMemcpyHostToDevice, s));
  const int tiles = (n + 15) / 16;
  int blocks = (tiles + 7) / 8;
  if (blocks > 1184) blocks = 1184;
  k_mlp_infer<<<blocks, 256, 0, s>>>(n, m->d_x, m->d_wb, m->d_master, m->d_norm, m->d_out);
  MLP_CUDA(m, cudaGetLastError());
  MLP_CUDA(m, cudaMemcpyAsync(y, m->d_out, sizeof(float) * NO * (size_t)n, cudaMemcpyDeviceToHost, s));
  MLP_CUDA(m, cudaStreamSynchronize(s));
  return ICF_OK;
}

int icf_mlp_forward_trace(icf_mlp *m, int n, const float *x, float *z1, float *h1, float *z2, float *h2, float *y) {
  if (!m || n <= 0 || !x || !z1 || !h1 || !z2 || !h2 || !y) return ICF_ERR_ARG;
  MLP_CUDA(m, cudaSetDevice(m->device));
  if (ensure_cap(m, n)) return ICF_ERR_CUDA;
  cudaStream_t s = m->stream;
  MLP_CUDA(m, cudaMemcpyAsync(m->d_x, x, sizeof(float) * NI * (size_t)n, cudaMemcpyHostToDevice, s));
  const int tiles = (n + 15) / 16;
  // the training forward writes the activations (no target: dy untouched)
  k_mlp_fwd_train<<<(tiles + 7) / 8, 256, 0, s>>>(n, m->d_x, nullptr, m->d_wb, m->d_master, m->d_norm, m->d_z1,
                                                  m->d_h1, m->d_z2, m->d_h2, m->d_dy, m->d_loss + 1);
  int blocks = (tiles + 7) / 8;
  if (blocks > 1184) blocks = 1184;
  k_mlp_infer<<<blocks, 256, 0, s>>>(n, m->d_x, m->d_wb, m->d_master, m->d_norm, m->d_out);
  MLP_CUDA(m, cudaGetLastError());
  const size_t hb = sizeof(float) * NH * (size_t)n;
  MLP_CUDA(m, cudaMemcpyAsync(z1, m->d_z1, hb, cudaMemcpyDeviceToHost, s));
  MLP_CUDA(m, cudaMemcpyAsync(h1, m->d_h1, hb, cudaMemcpyDeviceToHost, s));
  MLP_CUDA(m, cudaMemcpyAsync(z2, m->d_z2, hb, cudaMemcpyDeviceToHost, s));
  MLP_CUDA(m, cudaMemcpyAsync(h2, m->d_h2, hb, cudaMemcpyDeviceToHost, s));
  MLP_CUDA(m, cudaMemcpyAsync(y, m->d_out, sizeof(float) * NO * (size_t)n, cudaMemcpyDeviceToHost, s));
  MLP_CUDA(m, cudaStreamSynchronize(s));
  return ICF_OK;
}

int icf_mlp_grad(icf_mlp *m, int n, const float *x, const float *y, float *grad, float *loss) {
  if (!m || n <= 0 || !x || !y || !grad) return ICF_ERR_ARG;
  MLP_CUDA(m, cudaSetDevice(m->device));
  if (ensure_cap(m, n)) return ICF_ERR_CUDA;
  cudaStream_t s = m->stream;
  MLP_CUDA(m, cudaMemcpyAsync(m->d_x, x, sizeof(float) * NI * (size_t)n, cudaMemcpyHostToDevice, s));
  MLP_CUDA(m, cudaMemcpyAsync(m->d_y, y, sizeof(float) * NO * (size_t)n, cudaMemcpyHostToDevice, s));
  float l = 0.f;
  if (grad_on_device(m, n, &l)) return ICF_ERR_CUDA;
  MLP_CUDA(m, cudaMemcpy(grad, m->d_grad, sizeof(float) * NPAR, cudaMemcpyDeviceToHost));
  if (loss) *loss = l;
  return ICF_OK;
}

int icf_mlp_grad_dy(icf_mlp *m, int n, const float *x, const float *dy, float *grad) {
  if (!m || n <= 0 || !x || !dy) return ICF_ERR_ARG;
  MLP_CUDA(m, cudaSetDevice(m->device));
  if (ensure_cap(m, n)) return ICF_ERR_CUDA;
  cudaStream_t s = m->stream;
  MLP_CUDA(m, cudaMemcpyAsync(m->d_x, x, sizeof(float) * NI * (size_t)n, cudaMemcpyHostToDevice, s));
  MLP_CUDA(m, cudaMemcpyAsync(m->d_dy, dy, sizeof(float) * NO * (size_t)n, cudaMemcpyHostToDevice, s));
  if (grad_on_device(m, n, nullptr, true)) return ICF_ERR_CUDA;
  if (grad) MLP_CUDA(m, cudaMemcpyAsync(grad, m->d_grad, sizeof(float) * NPAR, cudaMemcpyDeviceToHost, s));
  MLP_CUDA(m, cudaStreamSynchronize(s));
  return ICF_OK;
}

int icf_mlp_adam_step(icf_mlp *m, const float *grad, float lr) {
  if (!m || !(lr > 0)) return ICF_ERR_ARG;
  MLP_CUDA(m, cudaSetDevice(m->device));
  cudaStream_t s = m->stream;
  if (grad) MLP_CUDA(m, cudaMemcpyAsync(m->d_grad, grad, sizeof(float) * NPAR, cudaMemcpyHostToDevice, s));
  m->adam_t++;
  const float b1c = 1.f - powf(0.9f, (float)m->adam_t), b2c = 1.f - powf(0.999f, (float)m->adam_t);
  k_mlp_adam<<<icf_blocks(NPAR, 256), 256, 0, s>>>(m->d_master, m->d_m, m->d_v, m->d_grad, lr, b1c, b2c);
  k_mlp_pack<<<icf_blocks(WB_N, 256), 256, 0, s>>>(m->d_master, m->d_wb);
  MLP_CUDA(m, cudaGetLastError());
  MLP_CUDA(m, cudaStreamSynchronize(s));
  return ICF_OK;
}

int icf_mlp_train(icf_mlp *m, int n, const float *x, const float *y, int epochs, int batch, float lr,
                  unsigned long long seed, float *loss_out) {
  if (!m || n <= 0 || !x || !y || epochs < 1 || batch < 16 || !(lr > 0)) return ICF_ERR_ARG;
  MLP_CUDA(m, cudaSetDevice(m->device));
  if (batch > n) batch = n;
  if (ensure_cap(m, batch)) return ICF_ERR_CUDA;
  cudaStream_t s = m->stream;
  // whole data set on the device, shuffled per epoch on the host (seeded)
  float *dx_all = nullptr, *dy_all = nullptr;
  int *d_order = nullptr;
  MLP_CUDA(m, cudaMalloc(&dx_all, sizeof(float) * NI * (size_t)n));
  MLP_CUDA(m, cudaMalloc(&dy_all, sizeof(float) * NO * (size_t)n));
  MLP_CUDA(m, cudaMalloc(&d_order, sizeof(int) * (size_t)n));
  MLP_CUDA(m, cudaMemcpy(dx_all, x, sizeof(float) * NI * (size_t)n, cudaMemcpyHostToDevice));
  MLP_CUDA(m, cudaMemcpy(dy_all, y, sizeof(float) * NO * (size_t)n, cudaMemcpyHostToDevice));
  std::vector<int> order(n);
  for (int i = 0; i < n; i++) order[i] = i;
  unsigned long long st = seed * 6364136223846793005ull + 1442695040888963407ull;
  float last = 0.f;
  int rc = ICF_OK;
  for (int ep = 0; ep < epochs && rc == ICF_OK; ep++) {
    for (int i = n - 1; i > 0; i--) {  // Fisher-Yates with a 64-bit LCG
      st = st * 6364136223846793005ull + 1442695040888963407ull;
      const int j = (int)((st >> 33) % (unsigned long long)(i + 1));
      std::swap(order[i], order[j]);
    }
    if (cudaMemcpyAsync(d_order, order.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, s) !=
        cudaSuccess) {
      rc = fail(m, ICF_ERR_CUDA, "order upload failed");
      break;
    }
    // contiguous batches of the shuffled order, gathered on the device
    for (int b0 = 0; b0 + batch <= n && rc == ICF_OK; b0 += batch) {
      k_gather_rows<<<icf_blocks(batch, 256), 256, 0, s>>>(batch, d_order + b0, dx_all, dy_all, m->d_x, m->d_y);
      rc = grad_on_device(m, batch, nullptr);
      if (rc) break;
      m->adam_t++;
      const float b1c = 1.f - powf(0.9f, (float)m->adam_t), b2c = 1.f - powf(0.999f, (float)m->adam_t);
      k_mlp_adam<<<icf_blocks(NPAR, 256), 256, 0, s>>>(m->d_master, m->d_m, m->d_v, m->d_grad, lr, b1c, b2c);
      k_mlp_pack<<<icf_blocks(WB_N, 256), 256, 0, s>>>(m->d_master, m->d_wb);
    }
    if (rc == ICF_OK && cudaGetLastError() != cudaSuccess) rc = fail(m, ICF_ERR_CUDA, "training launch failed");
  }
  if (rc == ICF_OK) {
    // loss over the whole set with the final weights (first `cap` nodes per pass)
    double tot = 0;
    for (int b0 = 0; b0 < n && rc == ICF_OK; b0 += m->cap) {
      const int k = std::min(m->cap, n - b0);
      cudaMemcpyAsync(m->d_x, dx_all + (size_t)b0 * NI, sizeof(float) * NI * (size_t)k, cudaMemcpyDeviceToDevice, s);
      cudaMemcpyAsync(m->d_y, dy_all + (size_t)b0 * NO, sizeof(float) * NO * (size_t)k, cudaMemcpyDeviceToDevice, s);
      float l = 0;
      rc = grad_on_device(m, k, &l);
      tot += (double)l * k;
    }
    last = (float)(tot / n);
  }
  cudaStreamSynchronize(s);  // the host order buffer is reused by the next epoch's upload only after this
  cudaFree(dx_all);
  cudaFree(dy_all);
  cudaFree(d_order);
  if (rc) return rc;
  if (loss_out) *loss_out = last;
  return ICF_OK;
}

}  // extern "C"
