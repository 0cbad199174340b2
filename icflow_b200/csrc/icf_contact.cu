// icf_contact.cu -- narrow phase, closest face and penalty contact.
//
// This file is compiled with -fmad=false: every product and sum is rounded on
// its own, in the order written, so the integer outputs that hinge on
// floating-point comparisons (the 8-bit inclusion masks, the closest face,
// the Voronoi region of the point-triangle distance) are reproducible bit for
// bit against a CPU evaluation with the same operation order.
//
//   k_narrow      kNarrowPhase_new (collision_kernels9/narrowphase.h:46-155)
//   k_expand      the host set expansion of GPU_Functionality.cs:566-580,
//                 done on the device as keys (node << 32 | element)
//   k_closest     kFindClosestFace (narrowphase.h:159-201) with dtn
//                 (dist_node2tri.h:14-129)
// The penalty response of the impacts (kCollisionResponseForce) is in
// icf_contact_deriv.cu, its region decision in icf_ptri.cuh.
#include <cub/cub.cuh>

#include "icf_collide.cuh"
#include "icf_internal.cuh"

namespace {

// ---- narrow phase (tet_inverse, tet_contains: icf_collide.cuh) ----------------
__global__ void k_narrow(int np, const int *__restrict__ pairs,
                         const int4 *__restrict__ selem,
                         const double4 *__restrict__ xc, int *__restrict__ masks,
                         int *__restrict__ counts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const int4 A = selem[pairs[2 * i]], B = selem[pairs[2 * i + 1]];
  const int na[4] = {A.x, A.y, A.z, A.w}, nb[4] = {B.x, B.y, B.z, B.w};
  int m = 0;
  bool shared = false;
  for (int p = 0; p < 4; p++)
    for (int q = 0; q < 4; q++) shared |= (na[p] == nb[q]);
  if (!shared) {
    double xa[12], xb[12];
    for (int k = 0; k < 4; k++) {
      const double4 pa = xc[na[k]], pb = xc[nb[k]];
      xa[3 * k] = pa.x; xa[3 * k + 1] = pa.y; xa[3 * k + 2] = pa.z;
      xb[3 * k] = pb.x; xb[3 * k + 1] = pb.y; xb[3 * k + 2] = pb.z;
    }
    double ba[9], bb[9];
    tet_inverse(xa, ba);
    tet_inverse(xb, bb);
    for (int k = 0; k < 4; k++)
      if (tet_contains(ba, xb[3 * k] - xa[0], xb[3 * k + 1] - xa[1], xb[3 * k + 2] - xa[2]))
        m |= 1 << k;
    for (int k = 0; k < 4; k++)
      if (tet_contains(bb, xa[3 * k] - xb[0], xa[3 * k + 1] - xb[1], xa[3 * k + 2] - xb[2]))
        m |= 16 << k;
  }
  masks[i] = m;
  counts[i] = __popc(m);
}

// (node << 32 | element) for every set bit; bit k < 4: vertex k of the second
// element is inside the first; bit 4+k: vertex k of the first inside the second.
__global__ void k_expand(int np, const int *__restrict__ pairs,
                         const int4 *__restrict__ selem, const int *__restrict__ masks,
                         const int *__restrict__ off, int eb,
                         unsigned long long *__restrict__ keys) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const int m = masks[i];
  if (!m) return;
  const int ea = pairs[2 * i], eb_ = pairs[2 * i + 1];
  const int4 A = selem[ea], B = selem[eb_];
  const int na[4] = {A.x, A.y, A.z, A.w}, nb[4] = {B.x, B.y, B.z, B.w};
  int w = off[i];
  for (int k = 0; k < 4; k++)
    if (m & (1 << k)) keys[w++] = ((unsigned long long)(unsigned)nb[k] << eb) | (unsigned)ea;
  for (int k = 0; k < 4; k++)
    if (m & (16 << k)) keys[w++] = ((unsigned long long)(unsigned)na[k] << eb) | (unsigned)eb_;
}

__device__ double clamp01(double n) { return n <= 0 ? 0 : n >= 1 ? 1 : n; }

// dtn, dist_node2tri.h:14-129 (including its clamp of -e/c in region 6)
__device__ double dtn(const double f[9], const double p[3]) {
  double E0[3], E1[3], v0[3];
  for (int k = 0; k < 3; k++) {
    E0[k] = f[3 + k] - f[k];
    E1[k] = f[6 + k] - f[k];
    v0[k] = f[k] - p[k];
  }
  const double a = E0[0] * E0[0] + E0[1] * E0[1] + E0[2] * E0[2];
  const double b = E0[0] * E1[0] + E0[1] * E1[1] + E0[2] * E1[2];
  const double c = E1[0] * E1[0] + E1[1] * E1[1] + E1[2] * E1[2];
  const double d = E0[0] * v0[0] + E0[1] * v0[1] + E0[2] * v0[2];
  const double e = E1[0] * v0[0] + E1[1] * v0[1] + E1[2] * v0[2];
  const double det = a * c - b * b;
  double s = b * e - c * d, t = b * d - a * e;
  if (s + t < det) {
    if (s < 0) {
      if (t < 0 && d < 0) { s = clamp01(-d / a); t = 0; }
      else { s = 0; t = clamp01(-e / c); }
    } else if (t < 0) {
      s = clamp01(-d / a);
      t = 0;
    } else {
      const double inv = 1.0 / det;
      s *= inv;
      t *= inv;
    }
  } else {
    if (s < 0) {
      const double t0 = b + d, t1 = c + e;
      if (t1 > t0) { s = clamp01((t1 - t0) / (a - 2 * b + c)); t = 1 - s; }
      else { t = clamp01(-e / c); s = 0; }
    } else if (t < 0) {
      if (a + d > b + e) { s = clamp01((c + e - b - d) / (a - 2 * b + c)); t = 1 - s; }
      else { s = clamp01(-e / c); t = 0; }
    } else {
      s = clamp01((c + e - b - d) / (a - 2 * b + c));
      t = 1 - s;
    }
  }
  double r = 0;
  for (int k = 0; k < 3; k++) {
    const double dk = f[k] + s * E0[k] + t * E1[k] - p[k];
    r += dk * dk;
  }
  return r;
}

// Eight threads per (node, element) key, each taking every eighth adjacent
// face; the group keeps the smallest distance, the first face in list order
// on ties (kFindClosestFace's strict minimum over the list in order).
__global__ void k_closest(int n, const int *__restrict__ n_dev, int eb, const unsigned long long *__restrict__ keys,
                          const int *__restrict__ adj_off, const int *__restrict__ adj,
                          const int *__restrict__ faces, const double4 *__restrict__ xc,
                          int4 *__restrict__ imp) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int i = (int)(t >> 3), g = (int)(t & 7);
  const bool valid = i < n && i < *n_dev;
  int node = 0, best = 0x7fffffff;
  double bestd = 0;
  bool have = false;
  if (valid) {
    const unsigned long long key = keys[i];
    node = (int)(key >> eb);
    const int el = (int)(key & ((1ull << eb) - 1));
    const double4 pp = xc[node];
    const double p[3] = {pp.x, pp.y, pp.z};
    for (int q = adj_off[el] + g; q < adj_off[el + 1]; q += 8) {
      const int fc = adj[q];
      double fx[9];
      for (int v = 0; v < 3; v++) {
        const double4 c = xc[faces[3 * fc + v]];
        fx[3 * v] = c.x; fx[3 * v + 1] = c.y; fx[3 * v + 2] = c.z;
      }
      const double dd = dtn(fx, p);
      if (!have || dd < bestd) {
        best = q;
        bestd = dd;
        have = true;
      }
    }
  }
  // (distance, list position) minimum over the group; lanes without a face
  // (or past the keys) take part with the largest position
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) {
    const double od = __shfl_xor_sync(0xffffffffu, bestd, o);
    const int oq = __shfl_xor_sync(0xffffffffu, best, o);
    const bool oh = __shfl_xor_sync(0xffffffffu, (int)have, o) != 0;
    if (oh && (!have || od < bestd || (od == bestd && oq < best))) {
      bestd = od;
      best = oq;
      have = true;
    }
  }
  if (!valid || g != 0) return;
  if (!have) {
    imp[i] = make_int4(node, -1, -1, -1);
    return;
  }
  const int fc = adj[best];
  imp[i] = make_int4(node, faces[3 * fc], faces[3 * fc + 1], faces[3 * fc + 2]);
}

// flag[0] = 1 unless the new list (n_dev[0] impacts) equals the n_built
// impacts the current structure was built from
__global__ void k_imp_same(int cap, const int *__restrict__ n_dev, int n_built, const int4 *__restrict__ a,
                           const int4 *__restrict__ b, int *__restrict__ flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = *n_dev;
  if (i == 0 && n != n_built) *flag = 1;
  if (i >= cap || i >= n || i >= n_built) return;
  const int4 x = a[i], y = b[i];
  if (x.x != y.x || x.y != y.y || x.z != y.z || x.w != y.w) *flag = 1;
}

}  // namespace

int icf_launch_imp_unit(icf_ctx *ctx, cudaStream_t stream) {
  const int rc = icf_launch_imp_deriv(ctx, stream);
  // ids, their rows and four node positions in; up to ten 96 B records, the
  // 64 B position map and a 96 B force record per impact
  icf_prof_mark(ctx, stream, "k_imp_deriv", (16LL + 16 + 128 + 64 + 96 + 8LL * ICF_IMP_REC * 10) * ctx->n_imp);
  return rc;
}

// Narrow phase + set expansion + closest face.  Leaves ctx->d_imp /
// ctx->n_imp set; the pattern must be rebuilt afterwards.  Two
// synchronisations (the expanded tuple count, which sizes the sort, and the
// result); the buffers are the context's workspace.  The new list is also
// compared, on the device, with the list the current structure was built
// from, so that the structure request that follows needs no round trip.
template <typename T>
static int grow_buf(icf_ctx *ctx, T **p, long long n) {
  cudaFree(*p);
  *p = nullptr;
  ICF_CUDA(ctx, cudaMalloc(p, sizeof(T) * (size_t)(n > 0 ? n : 1)));
  return ICF_OK;
}

int icf_run_narrow_phase(icf_ctx *ctx, int n_pairs, int *n_impacts) {
  cudaStream_t s = ctx->stream;
  icf_contact_ws &W = ctx->cws;
  ctx->imp_cmp_valid = false;
  if (n_pairs == 0) {
    ctx->n_imp = 0;
    *n_impacts = 0;
    return ICF_OK;
  }
  if (!W.d_small) ICF_CUDA(ctx, cudaMalloc(&W.d_small, 8 * sizeof(int)));
  if (!W.h_small) ICF_CUDA(ctx, cudaMallocHost(&W.h_small, 8 * sizeof(int)));
  if (n_pairs + 1LL > W.ncnt_cap) {
    ICF_TRY_RC(grow_buf(ctx, &W.ncnt, n_pairs + 1LL));
    ICF_TRY_RC(grow_buf(ctx, &W.noff, n_pairs + 1LL));
    W.ncnt_cap = n_pairs + 1LL;
  }
  // counts and offsets of the set bits
  k_narrow<<<icf_blocks(n_pairs, 128), 128, 0, s>>>(n_pairs, ctx->d_pairs, ctx->d_selem, ctx->d_xc,
                                                   ctx->d_masks, W.ncnt);
  ICF_CUDA(ctx, cudaGetLastError());
  ICF_CUDA(ctx, cudaMemsetAsync(W.ncnt + n_pairs, 0, sizeof(int), s));
  size_t tb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb, W.ncnt, W.noff, n_pairs + 1, s);
  if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
  ICF_CUDA(ctx, cub::DeviceScan::ExclusiveSum(ctx->d_tmp, tb, W.ncnt, W.noff, n_pairs + 1, s));
  ICF_CUDA(ctx, cudaMemcpyAsync(W.h_small + 4, W.noff + n_pairs, sizeof(int), cudaMemcpyDeviceToHost, s));
  ICF_CUDA(ctx, cudaStreamSynchronize(s));
  const int total = W.h_small[4];
  int eb = 1, vb = 1;
  while ((1LL << eb) < (long long)ctx->n_surf) eb++;
  while ((1LL << vb) < (long long)ctx->n_nodes) vb++;
  if (total > 0) {
    if (total > W.nkey_cap) {
      const long long c = total + total / 4 + 64;
      ICF_TRY_RC(grow_buf(ctx, &W.nk0, c));
      ICF_TRY_RC(grow_buf(ctx, &W.nk1, c));
      W.nkey_cap = c;
    }
    // keys node << eb | element, over the bits the ids need
    k_expand<<<icf_blocks(n_pairs, 128), 128, 0, s>>>(n_pairs, ctx->d_pairs, ctx->d_selem, ctx->d_masks, W.noff,
                                                     eb, W.nk0);
    tb = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, tb, W.nk0, W.nk1, total, 0, eb + vb, s);
    if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
    ICF_CUDA(ctx, cub::DeviceRadixSort::SortKeys(ctx->d_tmp, tb, W.nk0, W.nk1, total, 0, eb + vb, s));
    tb = 0;
    cub::DeviceSelect::Unique(nullptr, tb, W.nk1, W.nk0, W.d_small, total, s);
    if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
    ICF_CUDA(ctx, cub::DeviceSelect::Unique(ctx->d_tmp, tb, W.nk1, W.nk0, W.d_small, total, s));
  }
  return icf_finish_impacts(ctx, W.nk0, total, W.d_small, eb, n_impacts);
}

// The impacts of sorted, unique keys (node << eb | element; at most `total`,
// their count in d_n on the device): closest face of each, the comparison
// with the list the current structure was built from, one synchronisation.
int icf_finish_impacts(icf_ctx *ctx, const unsigned long long *keys, int total, const int *d_n, int eb,
                       int *n_impacts) {
  cudaStream_t s = ctx->stream;
  icf_contact_ws &W = ctx->cws;
  const bool cmp = ctx->n_imp_built >= 0 && ctx->imp_gen == ctx->imp_gen_built;
  int nu = 0;
  if (total > 0) {
    // the impact list holds at most `total` entries
    if (total > ctx->imp_cap) {
      ICF_TRY_RC(grow_buf(ctx, &ctx->d_imp, 2LL * total));
      ctx->imp_cap = 2 * total;
      ctx->imp_gen++;
    }
    k_closest<<<icf_blocks(8LL * total, 128), 128, 0, s>>>(total, d_n, eb, keys, ctx->d_adj_off, ctx->d_adj,
                                                          ctx->d_faces, ctx->d_xc, ctx->d_imp);
    ICF_CUDA(ctx, cudaGetLastError());
    ICF_CUDA(ctx, cudaMemsetAsync(W.d_small + 1, 0, sizeof(int), s));
    if (cmp && ctx->imp_gen == ctx->imp_gen_built)
      k_imp_same<<<icf_blocks(total, 256), 256, 0, s>>>(total, d_n, ctx->n_imp_built, ctx->d_imp,
                                                       ctx->d_imp_built, W.d_small + 1);
    ICF_CUDA(ctx, cudaMemcpyAsync(W.h_small, d_n, sizeof(int), cudaMemcpyDeviceToHost, s));
    ICF_CUDA(ctx, cudaMemcpyAsync(W.h_small + 1, W.d_small + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    ICF_CUDA(ctx, cudaStreamSynchronize(s));
    nu = W.h_small[0];
    ctx->imp_cmp_valid = cmp && ctx->imp_gen == ctx->imp_gen_built;
    ctx->imp_differ = W.h_small[1];
  } else {
    ctx->imp_cmp_valid = cmp;
    ctx->imp_differ = ctx->n_imp_built != 0;
  }
  ctx->n_imp = nu;
  *n_impacts = nu;
  return ICF_OK;
}

// Impact units with caller-chosen buffers (allocation-free entry point).
int icf_launch_imp_unit_bufs(icf_ctx *ctx, const double4 *xc, double *ks, cudaStream_t stream) {
  return icf_launch_imp_deriv_bufs(ctx, xc, ks, stream);
}
