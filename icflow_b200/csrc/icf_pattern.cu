// icf_pattern.cu -- the upper-triangular 3x3-block sparsity pattern and the
// slot-sorted contribution lists, built on the device.
//
// Static part (elements and every CZ that is not failed when the pattern is
// first built; MeshCollection.cs:91-109, j >= i).  The reference never
// clears its static neighbour sets (CSRDictionary.ClearStatic has no
// caller), so the static pattern only grows: it is built once and kept.
// Dynamic part (impacts, ImplicitModel3.cs:177-196, j > i) is merged into it
// on every icf_create_structure call.  Columns ascend within a row
// (CSRDictionary.cs:90) and slots number the blocks row by row.
//
// Each candidate block (unit, a, b) is a 64-bit key (alt_a << 32 | alt_b)
// paired with a 32-bit contribution code.  A stable radix sort by key puts
// the contributions of every block next to each other, in unit order; the
// run heads are the slots.  That sorted code list is what k_gather walks.
#include <cub/cub.cuh>

#include "icf_internal.cuh"

namespace {
constexpr unsigned long long KMAX = ~0ull;

__global__ void k_cand_tet(int ne, const int4 *__restrict__ elem, const int *__restrict__ alt,
                           unsigned long long *__restrict__ key, uint32_t *__restrict__ code) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const int4 id = elem[e];
  const int nid[4] = {id.x, id.y, id.z, id.w};
  int al[4];
  for (int i = 0; i < 4; i++) al[i] = alt[nid[i]];
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) {
      const size_t o = 16 * (size_t)e + 4 * a + b;
      const bool ok = al[a] >= 0 && al[b] >= 0 && al[b] >= al[a];
      key[o] = ok ? (((unsigned long long)al[a] << 32) | (unsigned)al[b]) : KMAX;
      code[o] = icf_code_tet(ICF_KIND_TET, e, a, b);
    }
}

__global__ void k_cand_cz(int nc, const int *__restrict__ cz, const int *__restrict__ fail,
                          const int *__restrict__ alt, unsigned long long *__restrict__ key,
                          uint32_t *__restrict__ code) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  int al[6];
  for (int i = 0; i < 6; i++) al[i] = alt[cz[8 * c + i]];
  const bool live = fail[c] == 0;
  for (int a = 0; a < 6; a++)
    for (int b = 0; b < 6; b++) {
      const size_t o = 36 * (size_t)c + 6 * a + b;
      const bool ok = live && al[a] >= 0 && al[b] >= 0 && al[b] >= al[a];
      key[o] = ok ? (((unsigned long long)al[a] << 32) | (unsigned)al[b]) : KMAX;
      code[o] = icf_code_cz(c, a, b);
    }
}

// run heads of a sorted key array (KMAX excluded)
__global__ void k_heads(long long n, const unsigned long long *__restrict__ key, int *__restrict__ flag) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned long long k = key[i];
  flag[i] = (k != KMAX && (i == 0 || key[i - 1] != k)) ? 1 : 0;
}

__global__ void k_slots(long long n, const unsigned long long *__restrict__ key,
                        const int *__restrict__ flag, const int *__restrict__ incl,
                        unsigned long long *__restrict__ skey, int *__restrict__ off) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n || !flag[i]) return;
  const int s = incl[i] - 1;
  skey[s] = key[i];
  off[s] = (int)i;
}

__device__ __forceinline__ long long lower_bound_u64(const unsigned long long *a, long long n,
                                                     unsigned long long v) {
  long long lo = 0, hi = n;
  while (lo < hi) {
    const long long m = (lo + hi) >> 1;
    if (a[m] < v) lo = m + 1;
    else hi = m;
  }
  return lo;
}

__global__ void k_count_valid(long long n, const unsigned long long *__restrict__ key, long long *out) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *out = lower_bound_u64(key, n, KMAX);
}

__global__ void k_rows(int N, int nnz, const unsigned long long *__restrict__ key, int *__restrict__ rows) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r > N) return;
  rows[r] = (int)lower_bound_u64(key, nnz, (unsigned long long)r << 32);
}

__global__ void k_cols(int nnz, const unsigned long long *__restrict__ key, int *__restrict__ cols) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nnz) return;
  cols[s] = (int)(key[s] & 0xffffffffull);
}

__global__ void k_cand_dyn(int ni, const int4 *__restrict__ imp, const int *__restrict__ alt,
                           unsigned long long *__restrict__ key) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= ni) return;
  const int4 id = imp[u];
  const int nid[4] = {id.x, id.y, id.z, id.w};
  int al[4];
  for (int i = 0; i < 4; i++) al[i] = nid[i] >= 0 ? alt[nid[i]] : -1;
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) {
      const bool ok = al[a] >= 0 && al[b] >= 0 && al[b] > al[a];
      key[16 * (size_t)u + 4 * a + b] = ok ? (((unsigned long long)al[a] << 32) | (unsigned)al[b]) : KMAX;
    }
}

// keep dynamic keys that are new (not in the static pattern); flag rows that
// fall outside the pattern (the reference would throw there)
__global__ void k_dyn_new(int n, const unsigned long long *__restrict__ dkey,
                          const unsigned long long *__restrict__ skey, int nnz_s, int N,
                          int *__restrict__ keep, int *__restrict__ bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned long long k = dkey[i];
  int kp = 0;
  if (k != KMAX) {
    if ((int)(k >> 32) >= N) atomicOr(bad, 1);
    const long long p = lower_bound_u64(skey, nnz_s, k);
    kp = !(p < nnz_s && skey[p] == k);
  }
  keep[i] = kp;
}

__global__ void k_merge_static(int nnz_s, const unsigned long long *__restrict__ skey,
                               const unsigned long long *__restrict__ dkey, int nd,
                               unsigned long long *__restrict__ mkey, int *__restrict__ src,
                               int *__restrict__ s2m) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nnz_s) return;
  const long long p = i + lower_bound_u64(dkey, nd, skey[i]);
  mkey[p] = skey[i];
  src[p] = i;
  s2m[i] = (int)p;
}

__global__ void k_merge_dyn(int nd, const unsigned long long *__restrict__ dkey,
                            const unsigned long long *__restrict__ skey, int nnz_s,
                            unsigned long long *__restrict__ mkey, int *__restrict__ src,
                            int *__restrict__ dynpos) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nd) return;
  const long long p = j + lower_bound_u64(skey, nnz_s, dkey[j]);
  mkey[p] = dkey[j];
  src[p] = -1;
  dynpos[j] = (int)p;
}

// Per static slot: where its CZ codes start (tet codes come first in the
// stable order), and whether it is a diagonal block.  Diagonal slots are
// listed per row, off-diagonal slots are flagged for compaction.
__global__ void k_slot_meta(int nnz_s, const unsigned long long *__restrict__ skey,
                            const int *__restrict__ rc_off, const uint32_t *__restrict__ rc,
                            int *__restrict__ rc_mid, int *__restrict__ diag_of_row,
                            int *__restrict__ offflag) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nnz_s) return;
  const int b = rc_off[s], e = rc_off[s + 1];
  int m = b;
  while (m < e && (rc[m] >> 30) == ICF_KIND_TET) m++;
  rc_mid[s] = m;
  const unsigned long long k = skey[s];
  const int row = (int)(k >> 32), col = (int)(k & 0xffffffffull);
  if (row == col) diag_of_row[row] = s;
  offflag[s] = row != col;
}

// Gather descriptors {merged position, first tet code, first CZ code, end}:
// per row for the diagonal blocks (position -1 if the row has none) and per
// off-diagonal block.
__global__ void k_desc(int n, const int *__restrict__ slot_of, const int *__restrict__ rc_off,
                       const int *__restrict__ rc_mid, const int *__restrict__ s2m, int identity,
                       int4 *__restrict__ desc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int st = slot_of[i];
  if (st < 0) {
    desc[i] = make_int4(-1, 0, 0, 0);
    return;
  }
  desc[i] = make_int4(identity ? st : s2m[st], rc_off[st], rc_mid[st], rc_off[st + 1]);
}

// ---- sliced-ELL gather lists (see icf_sell) ---------------------------------
// sort key of unit i: its window, then its per-lane tet and CZ iteration counts
__global__ void k_sell_key(int n, int wl, int lanes, const int4 *__restrict__ desc,
                           uint32_t *__restrict__ key, int *__restrict__ idx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int4 d = desc[i];
  int mt = d.x >= 0 ? (d.z - d.y + lanes - 1) / lanes : 0;
  int mc = d.x >= 0 ? (d.w - d.z + lanes - 1) / lanes : 0;
  mt = mt < 255 ? mt : 255;
  mc = mc < 255 ? mc : 255;
  key[i] = (uint32_t)(i >> wl) << 16 | (uint32_t)mt << 8 | (uint32_t)mc;
  idx[i] = i;
}

// one warp per slice: iteration counts (the slice's maxima) and unit table
__global__ void k_sell_count(int n, int n_slices, int lanes, const int *__restrict__ perm,
                             const int4 *__restrict__ desc, int with_row, const int *__restrict__ row_of,
                             int4 *__restrict__ meta, int *__restrict__ cnt, int2 *__restrict__ unit) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= n_slices) return;
  const int per = 32 / lanes;
  const int j = lane / lanes, sub = lane % lanes;
  const int u = w * per + j;
  int mt = 0, mc = 0;
  int2 un = make_int2(-1, -1);
  if (u < n) {
    const int i = perm[u];
    const int4 d = desc[i];
    if (d.x >= 0) {
      mt = (d.z - d.y + lanes - 1) / lanes;
      mc = (d.w - d.z + lanes - 1) / lanes;
    }
    un = make_int2(d.x, with_row ? (row_of ? row_of[i] : i) : -1);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mt = max(mt, __shfl_xor_sync(0xffffffffu, mt, o));
    mc = max(mc, __shfl_xor_sync(0xffffffffu, mc, o));
  }
  if (sub == 0) unit[w * per + j] = un;
  if (lane == 0) {
    meta[w] = make_int4(0, mt, mc, 0);
    cnt[w] = 32 * (mt + mc);
  }
}

__global__ void k_sell_fill(int n, int n_slices, int lanes, const int *__restrict__ perm,
                            const int4 *__restrict__ desc, const int *__restrict__ off,
                            const uint32_t *__restrict__ rc, int4 *__restrict__ meta,
                            uint32_t *__restrict__ codes) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= n_slices) return;
  const int per = 32 / lanes;
  const int j = lane / lanes, sub = lane % lanes;
  const int u = w * per + j;
  int4 d = make_int4(-1, 0, 0, 0);
  if (u < n) d = desc[perm[u]];
  const int4 m = meta[w];
  const long long o = off[w];
  const int nt = d.x >= 0 ? d.z - d.y : 0, nc = d.x >= 0 ? d.w - d.z : 0;
  for (int k = 0; k < m.y; k++) {
    const int q = k * lanes + sub;
    codes[o + 32LL * k + lane] = q < nt ? rc[d.y + q] : ICF_CODE_PAD;
  }
  for (int k = 0; k < m.z; k++) {
    const int q = k * lanes + sub;
    codes[o + 32LL * (m.y + k) + lane] = q < nc ? rc[d.z + q] : ICF_CODE_PAD;
  }
  if (lane == 0) meta[w].x = (int)o;
}

// number of contribution codes of the off-diagonal slots
__global__ void k_off_codes(int n, const int *__restrict__ offflag, const int *__restrict__ rc_off,
                            unsigned long long *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long c = (i < n && offflag[i]) ? (unsigned long long)(rc_off[i + 1] - rc_off[i]) : 0ull;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

__global__ void k_iota(int n, int *__restrict__ a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = i;
}

// impact contributions keyed by their merged slot
// 1 where the touched slot is a static off-diagonal block (written by the
// off-diagonal gather), else 0; flag[n] = 0
__global__ void k_flag_off(int n, const int *__restrict__ slot, const unsigned long long *__restrict__ mkey,
                           const int *__restrict__ src, int identity, int *__restrict__ flag) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g > n) return;
  flag[g] = g < n && icf_off_static(mkey, src, identity, slot[g]) ? 1 : 0;
}

// the touched slots in k_imp_add's order, a stable partition: diagonal and
// contact-only blocks at [0, n_a), static off-diagonal ones at [n_a, n), each
// part in slot order (so a warp's records and blocks lie close together); per
// slot its record range, slot and rhs row (diagonal blocks), -1 (static
// off-diagonal blocks) or -2 (contact-only blocks, which k_imp_add writes
// rather than adds to).  pref: the exclusive prefix sum of k_flag_off's flags.
__global__ void k_split_off(int n, int n_a, const int *__restrict__ slot, const int *__restrict__ off,
                            const unsigned long long *__restrict__ mkey, const int *__restrict__ pref,
                            int2 *__restrict__ range, int *__restrict__ pslot, int *__restrict__ row) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  const int sl = slot[g];
  const bool f = pref[g + 1] != pref[g];
  const int p = f ? n_a + pref[g] : g - pref[g];
  range[p] = make_int2(off[g], off[g + 1]);
  pslot[p] = sl;
  const unsigned long long k = mkey[sl];
  row[p] = (k >> 32) == (k & 0xffffffffull) ? (int)(k & 0xffffffffull) : (f ? -1 : -2);
}

__global__ void k_cand_imp_rc(int ni, const int4 *__restrict__ imp, const int *__restrict__ alt,
                              const unsigned long long *__restrict__ mkey, int nnz,
                              int *__restrict__ slot, uint32_t *__restrict__ code) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= ni) return;
  const int4 id = imp[u];
  const int nid[4] = {id.x, id.y, id.z, id.w};
  int al[4];
  for (int i = 0; i < 4; i++) al[i] = nid[i] >= 0 ? alt[nid[i]] : -1;
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) {
      const size_t o = 16 * (size_t)u + 4 * a + b;
      int s = 0x7fffffff;
      if (al[a] >= 0 && al[b] >= 0 && al[b] >= al[a]) {
        const unsigned long long k = ((unsigned long long)al[a] << 32) | (unsigned)al[b];
        const long long p = lower_bound_u64(mkey, nnz, k);
        if (p < nnz && mkey[p] == k) s = (int)p;
      }
      slot[o] = s;
      code[o] = icf_code_tet(ICF_KIND_IMP, u, a, b);
    }
}

// pos[16 u + 4 a + b] = position of impact code (u, a, b) in the slot-sorted
// list, for the valid codes (those before the invalid-slot run)
__global__ void k_imp_pos(int n, const int *__restrict__ n_valid, const uint32_t *__restrict__ code,
                          int *__restrict__ pos) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n || q >= *n_valid) return;
  const uint32_t c = code[q];
  pos[16 * (size_t)((c >> 4) & 0x3FFFFFFu) + (c & 15u)] = q;
}

// node incidence lists: (node, unit << 2 | vertex)
__global__ void k_node_inc_tet(int ne, const int4 *__restrict__ elem, int *__restrict__ node,
                               int *__restrict__ code) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const int4 id = elem[e];
  const int nid[4] = {id.x, id.y, id.z, id.w};
  for (int a = 0; a < 4; a++) {
    node[4 * (size_t)e + a] = nid[a];
    code[4 * (size_t)e + a] = (e << 2) | a;
  }
}
__global__ void k_node_inc_imp(int ni, const int4 *__restrict__ imp, int *__restrict__ node,
                               int *__restrict__ code) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= ni) return;
  const int4 id = imp[u];
  const int nid[4] = {id.x, id.y, id.z, id.w};
  for (int a = 0; a < 4; a++) {
    node[4 * (size_t)u + a] = nid[a] >= 0 ? nid[a] : 0x7fffffff;
    code[4 * (size_t)u + a] = (u << 2) | a;
  }
}
__global__ void k_offsets_from_sorted(int n_items, const int *__restrict__ node, int n_nodes,
                                      int *__restrict__ off) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > n_nodes) return;
  int lo = 0, hi = n_items;
  while (lo < hi) {
    const int m = (lo + hi) >> 1;
    if (node[m] < i) lo = m + 1;
    else hi = m;
  }
  off[i] = lo;
}

// pcsr maps in the reference's logical layout
__global__ void k_pcsr(int n, int k, const int *__restrict__ nodes, int stride,
                       const int *__restrict__ alt, const unsigned long long *__restrict__ mkey,
                       int nnz, int *__restrict__ out) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n) return;
  const int w = k * k + k;
  int al[6];
  for (int i = 0; i < k; i++) {
    const int nd = nodes[(size_t)u * stride + i];
    al[i] = nd >= 0 ? alt[nd] : -1;
  }
  for (int i = 0; i < k; i++) {
    for (int j = 0; j < k; j++) {
      int s = -1;
      if (al[i] >= 0 && al[j] >= 0 && al[j] >= al[i]) {
        const unsigned long long key = ((unsigned long long)al[i] << 32) | (unsigned)al[j];
        const long long p = lower_bound_u64(mkey, nnz, key);
        if (p < nnz && mkey[p] == key) s = (int)p;
      }
      out[(size_t)u * w + i * k + j] = s;
    }
    out[(size_t)u * w + k * k + i] = al[i];
  }
}

}  // namespace

template <typename T>
static int sort_pairs(icf_ctx *ctx, T *k_in, T *k_out, int *v_in, int *v_out, int n) {
  size_t tb = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, k_in, k_out, v_in, v_out, n, 0, (int)(8 * sizeof(T)),
                                  ctx->stream);
  if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
  ICF_CUDA(ctx, cub::DeviceRadixSort::SortPairs(ctx->d_tmp, tb, k_in, k_out, v_in, v_out, n, 0,
                                                (int)(8 * sizeof(T)), ctx->stream));
  return ICF_OK;
}

// node -> (unit, vertex) lists for the node forces
static int build_inc(icf_ctx *ctx, int n_items, void (*fill)(icf_ctx *, int *, int *),
                     icf_node_inc *out) {
  cudaStream_t s = ctx->stream;
  cudaFree(out->off);
  cudaFree(out->inc);
  out->off = out->inc = nullptr;
  ICF_CUDA(ctx, cudaMalloc(&out->off, sizeof(int) * (size_t)(ctx->n_nodes + 1)));
  ICF_CUDA(ctx, cudaMalloc(&out->inc, sizeof(int) * (size_t)(n_items > 0 ? n_items : 1)));
  if (n_items == 0) {
    ICF_CUDA(ctx, cudaMemsetAsync(out->off, 0, sizeof(int) * (size_t)(ctx->n_nodes + 1), s));
    return ICF_OK;
  }
  int *nd0, *nd1, *cd0;
  ICF_CUDA(ctx, cudaMallocAsync(&nd0, sizeof(int) * n_items, s));
  ICF_CUDA(ctx, cudaMallocAsync(&nd1, sizeof(int) * n_items, s));
  ICF_CUDA(ctx, cudaMallocAsync(&cd0, sizeof(int) * n_items, s));
  fill(ctx, nd0, cd0);
  ICF_CUDA(ctx, cudaGetLastError());
  int rc = sort_pairs<int>(ctx, nd0, nd1, cd0, out->inc, n_items);
  if (rc) return rc;
  k_offsets_from_sorted<<<icf_blocks(ctx->n_nodes + 1, 256), 256, 0, s>>>(n_items, nd1, ctx->n_nodes,
                                                                         out->off);
  ICF_CUDA(ctx, cudaGetLastError());
  ICF_CUDA(ctx, cudaFreeAsync(nd0, s));
  ICF_CUDA(ctx, cudaFreeAsync(nd1, s));
  ICF_CUDA(ctx, cudaFreeAsync(cd0, s));
  return ICF_OK;
}

static void fill_tet(icf_ctx *ctx, int *node, int *code) {
  k_node_inc_tet<<<icf_blocks(ctx->n_elem, 256), 256, 0, ctx->stream>>>(ctx->n_elem, ctx->d_elem, node,
                                                                       code);
}
static void fill_imp(icf_ctx *ctx, int *node, int *code) {
  k_node_inc_imp<<<icf_blocks(ctx->n_imp, 256), 256, 0, ctx->stream>>>(ctx->n_imp, ctx->d_imp, node, code);
}

int icf_get_node_inc(icf_ctx *ctx, icf_node_inc *tets, icf_node_inc *imps) {
  if (!ctx->tet_inc.off) {
    int rc = build_inc(ctx, 4 * ctx->n_elem, fill_tet, &ctx->tet_inc);
    if (rc) return rc;
  }
  // impact incidences are rebuilt whenever asked (impacts change per iteration)
  int rc = build_inc(ctx, 4 * ctx->n_imp, fill_imp, &ctx->imp_inc);
  if (rc) return rc;
  *tets = ctx->tet_inc;
  *imps = ctx->imp_inc;
  return ICF_OK;
}

int icf_build_static_pattern(icf_ctx *ctx) {
  cudaStream_t s = ctx->stream;
  const long long nc = 16LL * ctx->n_elem + 36LL * ctx->n_cz;
  if (nc >= (1LL << 31)) return icf_fail(ctx, ICF_ERR_SIZE, "pattern candidate count exceeds 2^31");
  if (nc == 0) {
    ctx->nnz_s = 0;
    ctx->n_rc = 0;
    ctx->N = 0;
    ICF_CUDA(ctx, cudaMalloc(&ctx->d_skeys, sizeof(unsigned long long)));
    ICF_CUDA(ctx, cudaMalloc(&ctx->d_rc_off, sizeof(int)));
    ICF_CUDA(ctx, cudaMemset(ctx->d_rc_off, 0, sizeof(int)));
    return ICF_OK;
  }
  unsigned long long *k0, *k1;
  uint32_t *c0;
  int *flag, *incl;
  long long *d_nv;
  ICF_CUDA(ctx, cudaMallocAsync(&k0, sizeof(unsigned long long) * (nc + 1), s));
  ICF_CUDA(ctx, cudaMallocAsync(&k1, sizeof(unsigned long long) * (nc + 1), s));
  ICF_CUDA(ctx, cudaMallocAsync(&c0, sizeof(uint32_t) * (nc + 1), s));
  ICF_CUDA(ctx, cudaMallocAsync(&flag, sizeof(int) * (nc + 1), s));
  ICF_CUDA(ctx, cudaMallocAsync(&incl, sizeof(int) * (nc + 1), s));
  ICF_CUDA(ctx, cudaMallocAsync(&d_nv, sizeof(long long), s));
  if (ctx->d_rc) cudaFree(ctx->d_rc);
  ctx->d_rc = nullptr;
  ICF_CUDA(ctx, cudaMalloc(&ctx->d_rc, sizeof(uint32_t) * (nc + 1)));
  if (ctx->n_elem)
    k_cand_tet<<<icf_blocks(ctx->n_elem, 256), 256, 0, s>>>(ctx->n_elem, ctx->d_elem, ctx->d_alt, k0, c0);
  if (ctx->n_cz)
    k_cand_cz<<<icf_blocks(ctx->n_cz, 256), 256, 0, s>>>(ctx->n_cz, ctx->d_cz, ctx->d_czfail, ctx->d_alt,
                                                        k0 + 16LL * ctx->n_elem, c0 + 16LL * ctx->n_elem);
  ICF_CUDA(ctx, cudaGetLastError());
  {
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, k0, k1, c0, ctx->d_rc, (int)nc, 0, 64, s);
    if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
    ICF_CUDA(ctx, cub::DeviceRadixSort::SortPairs(ctx->d_tmp, tb, k0, k1, c0, ctx->d_rc, (int)nc, 0, 64, s));
  }
  k_heads<<<icf_blocks(nc, 256), 256, 0, s>>>(nc, k1, flag);
  {
    size_t tb = 0;
    cub::DeviceScan::InclusiveSum(nullptr, tb, flag, incl, (int)nc, s);
    if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
    ICF_CUDA(ctx, cub::DeviceScan::InclusiveSum(ctx->d_tmp, tb, flag, incl, (int)nc, s));
  }
  int nnz_s = 0;
  long long nv = 0;
  k_count_valid<<<1, 32, 0, s>>>(nc, k1, d_nv);
  if (nc > 0) ICF_CUDA(ctx, cudaMemcpyAsync(&nnz_s, incl + nc - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
  ICF_CUDA(ctx, cudaMemcpyAsync(&nv, d_nv, sizeof(long long), cudaMemcpyDeviceToHost, s));
  ICF_CUDA(ctx, cudaStreamSynchronize(s));
  cudaFree(ctx->d_skeys);
  cudaFree(ctx->d_rc_off);
  ctx->d_skeys = nullptr;
  ctx->d_rc_off = nullptr;
  ICF_CUDA(ctx, cudaMalloc(&ctx->d_skeys, sizeof(unsigned long long) * (size_t)(nnz_s + 1)));
  ICF_CUDA(ctx, cudaMalloc(&ctx->d_rc_off, sizeof(int) * (size_t)(nnz_s + 1)));
  k_slots<<<icf_blocks(nc, 256), 256, 0, s>>>(nc, k1, flag, incl, ctx->d_skeys, ctx->d_rc_off);
  const int nvi = (int)nv;
  ICF_CUDA(ctx, cudaMemcpyAsync(ctx->d_rc_off + nnz_s, &nvi, sizeof(int), cudaMemcpyHostToDevice, s));
  unsigned long long last = 0;
  if (nnz_s > 0)
    ICF_CUDA(ctx, cudaMemcpyAsync(&last, ctx->d_skeys + nnz_s - 1, sizeof(last), cudaMemcpyDeviceToHost, s));
  ICF_CUDA(ctx, cudaFreeAsync(k0, s));
  ICF_CUDA(ctx, cudaFreeAsync(k1, s));
  ICF_CUDA(ctx, cudaFreeAsync(c0, s));
  ICF_CUDA(ctx, cudaFreeAsync(flag, s));
  ICF_CUDA(ctx, cudaFreeAsync(incl, s));
  ICF_CUDA(ctx, cudaFreeAsync(d_nv, s));
  ICF_CUDA(ctx, cudaStreamSynchronize(s));
  ctx->nnz_s = nnz_s;
  ctx->n_rc = nv;
  ctx->N = nnz_s > 0 ? (int)(last >> 32) + 1 : 0;

  // gather metadata: CZ-code start per slot, diagonal slot per row, the
  // compacted list of off-diagonal slots
  const int N = ctx->N;
  cudaFree(ctx->d_rc_mid);
  cudaFree(ctx->d_diag);
  cudaFree(ctx->d_offd);
  ctx->d_rc_mid = ctx->d_diag = ctx->d_offd = nullptr;
  ICF_CUDA(ctx, cudaMalloc(&ctx->d_rc_mid, sizeof(int) * (size_t)(nnz_s + 1)));
  ICF_CUDA(ctx, cudaMalloc(&ctx->d_diag, sizeof(int) * (size_t)(N + 1)));
  ICF_CUDA(ctx, cudaMalloc(&ctx->d_offd, sizeof(int) * (size_t)(nnz_s + 1)));
  ICF_CUDA(ctx, cudaMemsetAsync(ctx->d_diag, 0xff, sizeof(int) * (size_t)(N + 1), s));
  ctx->n_offd = 0;
  if (nnz_s > 0) {
    int *offflag, *iota, *d_n;
    ICF_CUDA(ctx, cudaMallocAsync(&offflag, sizeof(int) * nnz_s, s));
    ICF_CUDA(ctx, cudaMallocAsync(&iota, sizeof(int) * nnz_s, s));
    ICF_CUDA(ctx, cudaMallocAsync(&d_n, sizeof(int), s));
    k_slot_meta<<<icf_blocks(nnz_s, 256), 256, 0, s>>>(nnz_s, ctx->d_skeys, ctx->d_rc_off, ctx->d_rc,
                                                      ctx->d_rc_mid, ctx->d_diag, offflag);
    k_iota<<<icf_blocks(nnz_s, 256), 256, 0, s>>>(nnz_s, iota);
    ICF_CUDA(ctx, cudaGetLastError());
    size_t tb = 0;
    cub::DeviceSelect::Flagged(nullptr, tb, iota, offflag, ctx->d_offd, d_n, nnz_s, s);
    if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
    ICF_CUDA(ctx, cub::DeviceSelect::Flagged(ctx->d_tmp, tb, iota, offflag, ctx->d_offd, d_n, nnz_s, s));
    ICF_CUDA(ctx, cudaMemcpyAsync(&ctx->n_offd, d_n, sizeof(int), cudaMemcpyDeviceToHost, s));
    unsigned long long *d_c;
    ICF_CUDA(ctx, cudaMallocAsync(&d_c, sizeof(unsigned long long), s));
    ICF_CUDA(ctx, cudaMemsetAsync(d_c, 0, sizeof(unsigned long long), s));
    k_off_codes<<<icf_blocks(nnz_s, 256), 256, 0, s>>>(nnz_s, offflag, ctx->d_rc_off, d_c);
    unsigned long long n_off_codes = 0;
    ICF_CUDA(ctx, cudaMemcpyAsync(&n_off_codes, d_c, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    ICF_CUDA(ctx, cudaFreeAsync(d_c, s));
    ICF_CUDA(ctx, cudaFreeAsync(offflag, s));
    ICF_CUDA(ctx, cudaFreeAsync(iota, s));
    ICF_CUDA(ctx, cudaFreeAsync(d_n, s));
    ICF_CUDA(ctx, cudaStreamSynchronize(s));
    ctx->n_rc_off = (long long)n_off_codes;
  }
  return ICF_OK;
}

// total contribution codes of n descriptors
__global__ void k_real_codes(int n, const int4 *__restrict__ desc, unsigned long long *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long c = 0;
  if (i < n) {
    const int4 d = desc[i];
    if (d.x >= 0) c = (unsigned long long)(d.w - d.y);
  }
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

// Builds the sliced-ELL lists of a gather from its descriptors (n units).
static int build_sell(icf_ctx *ctx, const int4 *desc, int n, int wl, bool with_row, icf_sell *S,
                      cudaStream_t s, const int *row_of = nullptr) {
  const int per = 32 / S->lanes;
  S->n_units = n;
  S->n_slices = (n + per - 1) / per;
  S->n_codes = 0;
  S->n_real = 0;
  if (n == 0) return ICF_OK;
  const int ns = S->n_slices;
  if (ns > S->slices_cap || !S->meta) {
    cudaFree(S->meta);
    cudaFree(S->unit);
    cudaFree(S->unit_s);
    S->unit_s = nullptr;
    S->meta = nullptr;
    S->unit = nullptr;
    const int cap = ns + ns / 4 + 16;
    ICF_CUDA(ctx, cudaMalloc(&S->meta, sizeof(int4) * (size_t)cap));
    ICF_CUDA(ctx, cudaMalloc(&S->unit, sizeof(int2) * (size_t)cap * per));
    ICF_CUDA(ctx, cudaMalloc(&S->unit_s, sizeof(int2) * (size_t)cap * per));
    S->slices_cap = cap;
  }
  uint32_t *k0, *k1;
  int *i0, *perm, *cnt, *off;
  ICF_CUDA(ctx, cudaMallocAsync(&k0, sizeof(uint32_t) * (size_t)n, s));
  ICF_CUDA(ctx, cudaMallocAsync(&k1, sizeof(uint32_t) * (size_t)n, s));
  ICF_CUDA(ctx, cudaMallocAsync(&i0, sizeof(int) * (size_t)n, s));
  ICF_CUDA(ctx, cudaMallocAsync(&perm, sizeof(int) * (size_t)n, s));
  ICF_CUDA(ctx, cudaMallocAsync(&cnt, sizeof(int) * (size_t)(ns + 1), s));
  ICF_CUDA(ctx, cudaMallocAsync(&off, sizeof(int) * (size_t)(ns + 1), s));
  size_t tb = 0;
  if (S->natural) {
    k_iota<<<icf_blocks(n, 256), 256, 0, s>>>(n, perm);
  } else {
    k_sell_key<<<icf_blocks(n, 256), 256, 0, s>>>(n, wl, S->lanes, desc, k0, i0);
    int end_bit = 16;
    while ((((long long)n - 1) >> wl) >> (end_bit - 16)) end_bit++;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, k0, k1, i0, perm, n, 0, end_bit, s);
    if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
    ICF_CUDA(ctx, cub::DeviceRadixSort::SortPairs(ctx->d_tmp, tb, k0, k1, i0, perm, n, 0, end_bit, s));
  }
  ICF_CUDA(ctx, cudaMemsetAsync(S->unit_s, 0xff, sizeof(int2) * (size_t)ns * per, s));
  k_sell_count<<<icf_blocks(32LL * ns, 256), 256, 0, s>>>(n, ns, S->lanes, perm, desc, with_row ? 1 : 0, row_of,
                                                         S->meta, cnt, S->unit_s);
  ICF_CUDA(ctx, cudaMemsetAsync(cnt + ns, 0, sizeof(int), s));
  tb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, off, ns + 1, s);
  if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
  ICF_CUDA(ctx, cub::DeviceScan::ExclusiveSum(ctx->d_tmp, tb, cnt, off, ns + 1, s));
  unsigned long long *d_real;
  ICF_CUDA(ctx, cudaMallocAsync(&d_real, sizeof(unsigned long long), s));
  ICF_CUDA(ctx, cudaMemsetAsync(d_real, 0, sizeof(unsigned long long), s));
  k_real_codes<<<icf_blocks(n, 256), 256, 0, s>>>(n, desc, d_real);
  int total = 0;
  unsigned long long real = 0;
  ICF_CUDA(ctx, cudaMemcpyAsync(&total, off + ns, sizeof(int), cudaMemcpyDeviceToHost, s));
  ICF_CUDA(ctx, cudaMemcpyAsync(&real, d_real, sizeof(real), cudaMemcpyDeviceToHost, s));
  ICF_CUDA(ctx, cudaStreamSynchronize(s));
  ICF_CUDA(ctx, cudaFreeAsync(d_real, s));
  S->n_real = (long long)real;
  if (total < 0) return icf_fail(ctx, ICF_ERR_SIZE, "gather code list exceeds 2^31 entries");
  if (total > S->codes_cap || !S->codes) {
    cudaFree(S->codes);
    S->codes = nullptr;
    const long long cap = (long long)total + total / 4 + 32;
    ICF_CUDA(ctx, cudaMalloc(&S->codes, sizeof(uint32_t) * (size_t)cap));
    S->codes_cap = cap;
  }
  k_sell_fill<<<icf_blocks(32LL * ns, 256), 256, 0, s>>>(n, ns, S->lanes, perm, desc, off, ctx->d_rc, S->meta,
                                                        S->codes);
  ICF_CUDA(ctx, cudaGetLastError());
  S->n_codes = total;
  ICF_CUDA(ctx, cudaFreeAsync(k0, s));
  ICF_CUDA(ctx, cudaFreeAsync(k1, s));
  ICF_CUDA(ctx, cudaFreeAsync(i0, s));
  ICF_CUDA(ctx, cudaFreeAsync(perm, s));
  ICF_CUDA(ctx, cudaFreeAsync(cnt, s));
  ICF_CUDA(ctx, cudaFreeAsync(off, s));
  return ICF_OK;
}

// 1 for a descriptor with CZ codes
__global__ void k_has_cz(int n, const int4 *__restrict__ desc, int *__restrict__ flag, int *__restrict__ noflag,
                         int *__restrict__ idx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int4 d = desc[i];
  const int f = (d.x >= 0 && d.w > d.z) ? 1 : 0;
  flag[i] = f;
  noflag[i] = 1 - f;
  idx[i] = i;
}

// The gather lists of the current descriptors.  With split_cz (and the
// per-tet record layout) the units split into those without CZ codes
// (sell_off / sell_diag) and those with (sell_off_cz / sell_diag_cz); the
// diagonal lists carry each unit's row explicitly.
static int build_lists(icf_ctx *ctx, bool off, bool diag) {
  cudaStream_t s = ctx->stream;
  const bool split = ctx->split_cz && ctx->layout == ICF_LAYOUT_RECORDS && ctx->n_cz > 0;
  for (int k = 0; k < 2; k++) {
    if ((k == 0 && !off) || (k == 1 && !diag)) continue;
    const int4 *desc = k == 0 ? ctx->d_gdesc_off : ctx->d_gdesc_diag;
    const int n = k == 0 ? ctx->n_offd : ctx->N;
    icf_sell *A = k == 0 ? &ctx->sell_off : &ctx->sell_diag;
    icf_sell *B = k == 0 ? &ctx->sell_off_cz : &ctx->sell_diag_cz;
    const int wl = k == 0 ? 12 : (A->lanes >= 4 ? 10 : 11);
    if (!split || n == 0) {
      if (build_sell(ctx, desc, n, wl, k == 1, A, s)) return ICF_ERR_CUDA;
      B->n_units = B->n_slices = 0;
      B->n_codes = 0;
      continue;
    }
    int *flag, *noflag, *idx, *ia, *ib, *d_n;
    int4 *da, *db;
    ICF_CUDA(ctx, cudaMallocAsync(&flag, sizeof(int) * (size_t)n, s));
    ICF_CUDA(ctx, cudaMallocAsync(&noflag, sizeof(int) * (size_t)n, s));
    ICF_CUDA(ctx, cudaMallocAsync(&idx, sizeof(int) * (size_t)n, s));
    ICF_CUDA(ctx, cudaMallocAsync(&ia, sizeof(int) * (size_t)n, s));
    ICF_CUDA(ctx, cudaMallocAsync(&ib, sizeof(int) * (size_t)n, s));
    ICF_CUDA(ctx, cudaMallocAsync(&da, sizeof(int4) * (size_t)n, s));
    ICF_CUDA(ctx, cudaMallocAsync(&db, sizeof(int4) * (size_t)n, s));
    ICF_CUDA(ctx, cudaMallocAsync(&d_n, sizeof(int) * 4, s));
    k_has_cz<<<icf_blocks(n, 256), 256, 0, s>>>(n, desc, flag, noflag, idx);
    size_t tb = 0;
    cub::DeviceSelect::Flagged(nullptr, tb, desc, noflag, da, d_n, n, s);
    if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
    ICF_CUDA(ctx, cub::DeviceSelect::Flagged(ctx->d_tmp, tb, desc, noflag, da, d_n, n, s));
    ICF_CUDA(ctx, cub::DeviceSelect::Flagged(ctx->d_tmp, tb, desc, flag, db, d_n + 1, n, s));
    ICF_CUDA(ctx, cub::DeviceSelect::Flagged(ctx->d_tmp, tb, idx, noflag, ia, d_n + 2, n, s));
    ICF_CUDA(ctx, cub::DeviceSelect::Flagged(ctx->d_tmp, tb, idx, flag, ib, d_n + 3, n, s));
    int h_n[4] = {0, 0, 0, 0};
    ICF_CUDA(ctx, cudaMemcpyAsync(h_n, d_n, sizeof(h_n), cudaMemcpyDeviceToHost, s));
    ICF_CUDA(ctx, cudaStreamSynchronize(s));
    if (build_sell(ctx, da, h_n[0], wl, k == 1, A, s, k == 1 ? ia : nullptr)) return ICF_ERR_CUDA;
    if (build_sell(ctx, db, h_n[1], wl, k == 1, B, s, k == 1 ? ib : nullptr)) return ICF_ERR_CUDA;
    ICF_CUDA(ctx, cudaStreamSynchronize(s));
    void *tmp[] = {flag, noflag, idx, ia, ib, da, db, d_n};
    for (void *q : tmp) ICF_CUDA(ctx, cudaFreeAsync(q, s));
  }
  return ICF_OK;
}

template <typename T>
static int grow(icf_ctx *ctx, T **p, int *cap, long long n) {
  if (n <= *cap && *p) return ICF_OK;
  cudaFree(*p);
  *p = nullptr;
  const long long c = n + n / 4 + 16;
  ICF_CUDA(ctx, cudaMalloc(p, sizeof(T) * (size_t)c));
  *cap = (int)c;
  return ICF_OK;
}

int icf_build_merged_pattern(icf_ctx *ctx) {
  cudaStream_t s = ctx->stream;
  const int nnz_s = ctx->nnz_s, N = ctx->N;
  int nd = 0;
  unsigned long long *dkeys = nullptr;
  if (ctx->n_imp > 0) {
    const int n = 16 * ctx->n_imp;
    unsigned long long *a, *b;
    int *keep, *d_nd, *d_bad;
    ICF_CUDA(ctx, cudaMallocAsync(&a, sizeof(unsigned long long) * n, s));
    ICF_CUDA(ctx, cudaMallocAsync(&b, sizeof(unsigned long long) * n, s));
    ICF_CUDA(ctx, cudaMallocAsync(&keep, sizeof(int) * n, s));
    ICF_CUDA(ctx, cudaMallocAsync(&d_nd, sizeof(int) * 2, s));
    d_bad = d_nd + 1;
    ICF_CUDA(ctx, cudaMemsetAsync(d_nd, 0, sizeof(int) * 2, s));
    k_cand_dyn<<<icf_blocks(ctx->n_imp, 128), 128, 0, s>>>(ctx->n_imp, ctx->d_imp, ctx->d_alt, a);
    size_t tb = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, tb, a, b, n, 0, 64, s);
    if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
    ICF_CUDA(ctx, cub::DeviceRadixSort::SortKeys(ctx->d_tmp, tb, a, b, n, 0, 64, s));
    tb = 0;
    cub::DeviceSelect::Unique(nullptr, tb, b, a, d_nd, n, s);
    if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
    ICF_CUDA(ctx, cub::DeviceSelect::Unique(ctx->d_tmp, tb, b, a, d_nd, n, s));
    int nu = 0;
    ICF_CUDA(ctx, cudaMemcpyAsync(&nu, d_nd, sizeof(int), cudaMemcpyDeviceToHost, s));
    ICF_CUDA(ctx, cudaStreamSynchronize(s));
    if (nu > 0) k_dyn_new<<<icf_blocks(nu, 128), 128, 0, s>>>(nu, a, ctx->d_skeys, nnz_s, N, keep, d_bad);
    tb = 0;
    cub::DeviceSelect::Flagged(nullptr, tb, a, keep, b, d_nd, nu, s);
    if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
    ICF_CUDA(ctx, cub::DeviceSelect::Flagged(ctx->d_tmp, tb, a, keep, b, d_nd, nu, s));
    int hb[2] = {0, 0};
    ICF_CUDA(ctx, cudaMemcpyAsync(hb, d_nd, sizeof(int) * 2, cudaMemcpyDeviceToHost, s));
    ICF_CUDA(ctx, cudaStreamSynchronize(s));
    nd = hb[0];
    if (hb[1]) return icf_fail(ctx, ICF_ERR_STATE, "an impact references a row outside the pattern");
    dkeys = b;
    ICF_CUDA(ctx, cudaFreeAsync(a, s));
    ICF_CUDA(ctx, cudaFreeAsync(keep, s));
    ICF_CUDA(ctx, cudaFreeAsync(d_nd, s));
  }
  const int nnz = nnz_s + nd;
  if (nnz + 1 > ctx->cols_cap || !ctx->d_cols) {
    cudaFree(ctx->d_cols);
    cudaFree(ctx->d_src);
    cudaFree(ctx->d_mkeys);
    ctx->d_cols = ctx->d_src = nullptr;
    ctx->d_mkeys = nullptr;
    const long long cap = nnz + 1 + nnz / 8 + 64;
    ICF_CUDA(ctx, cudaMalloc(&ctx->d_cols, sizeof(int) * (size_t)cap));
    ICF_CUDA(ctx, cudaMalloc(&ctx->d_src, sizeof(int) * (size_t)cap));
    ICF_CUDA(ctx, cudaMalloc(&ctx->d_mkeys, sizeof(unsigned long long) * (size_t)cap));
    ctx->cols_cap = (int)cap;
  }
  int rc = grow(ctx, &ctx->d_rows, &ctx->rows_cap, (long long)N + 1);
  if (rc) return rc;
  if (nd == 0) {
    ICF_CUDA(ctx, cudaMemcpyAsync(ctx->d_mkeys, ctx->d_skeys, sizeof(unsigned long long) * (size_t)nnz_s,
                                  cudaMemcpyDeviceToDevice, s));
    ctx->src_identity = true;
  } else {
    // static -> merged positions and the positions of the contact-only blocks
    if (!ctx->d_s2m || ctx->s2m_cap < nnz_s + 1) {
      cudaFree(ctx->d_s2m);
      ctx->d_s2m = nullptr;
      ICF_CUDA(ctx, cudaMalloc(&ctx->d_s2m, sizeof(int) * (size_t)(nnz_s + 1)));
      ctx->s2m_cap = nnz_s + 1;
    }
    if (!ctx->d_dynpos || ctx->dynpos_cap < nd) {
      cudaFree(ctx->d_dynpos);
      ctx->d_dynpos = nullptr;
      ICF_CUDA(ctx, cudaMalloc(&ctx->d_dynpos, sizeof(int) * (size_t)(2 * nd)));
      ctx->dynpos_cap = 2 * nd;
    }
    if (nnz_s > 0)
      k_merge_static<<<icf_blocks(nnz_s, 256), 256, 0, s>>>(nnz_s, ctx->d_skeys, dkeys, nd, ctx->d_mkeys,
                                                           ctx->d_src, ctx->d_s2m);
    k_merge_dyn<<<icf_blocks(nd, 256), 256, 0, s>>>(nd, dkeys, ctx->d_skeys, nnz_s, ctx->d_mkeys, ctx->d_src,
                                                   ctx->d_dynpos);
    ctx->src_identity = false;
  }
  ctx->n_dyn = nd;
  // gather descriptors for this merge
  if (!ctx->d_gdesc_diag || ctx->gdesc_cap < N + ctx->n_offd + 2) {
    cudaFree(ctx->d_gdesc_diag);
    ctx->d_gdesc_diag = nullptr;
    ICF_CUDA(ctx, cudaMalloc(&ctx->d_gdesc_diag, sizeof(int4) * (size_t)(N + ctx->n_offd + 2)));
    ctx->gdesc_cap = N + ctx->n_offd + 2;
  }
  ctx->d_gdesc_off = ctx->d_gdesc_diag + N + 1;
  // the gather lists depend on the static pattern only: built once, in
  // static slots, then mapped to the merged slots of every structure
  if (!ctx->lists_static) {
    if (N > 0)
      k_desc<<<icf_blocks(N, 256), 256, 0, s>>>(N, ctx->d_diag, ctx->d_rc_off, ctx->d_rc_mid, nullptr, 1,
                                               ctx->d_gdesc_diag);
    if (ctx->n_offd > 0)
      k_desc<<<icf_blocks(ctx->n_offd, 256), 256, 0, s>>>(ctx->n_offd, ctx->d_offd, ctx->d_rc_off,
                                                         ctx->d_rc_mid, nullptr, 1, ctx->d_gdesc_off);
    ctx->sell_off.lanes = ctx->sell_off_cz.lanes = 1;
    ctx->sell_off.natural = ctx->sell_off_cz.natural = icf_gather_variant_natural(ctx->tune_off);
    ctx->sell_diag.lanes = ctx->sell_diag_cz.lanes = icf_gather_variant_lanes(ctx->tune_diag);
    if (build_lists(ctx, true, true)) return ICF_ERR_CUDA;
    if (icf_build_contrib(ctx)) return ICF_ERR_CUDA;
    ctx->lists_static = true;
  }
  if (icf_remap_lists(ctx)) return ICF_ERR_CUDA;
  if (ctx->tiles.built && icf_remap_tiles(ctx)) return ICF_ERR_CUDA;
  if (dkeys) ICF_CUDA(ctx, cudaFreeAsync(dkeys, s));
  if (nnz > 0) k_cols<<<icf_blocks(nnz, 256), 256, 0, s>>>(nnz, ctx->d_mkeys, ctx->d_cols);
  k_rows<<<icf_blocks((long long)N + 1, 256), 256, 0, s>>>(N, nnz, ctx->d_mkeys, ctx->d_rows);
  ICF_CUDA(ctx, cudaGetLastError());
  ctx->nnz = nnz;

  // impact contributions grouped by slot
  ctx->n_crs = 0;
  ctx->n_crs_off = 0;
  if (ctx->n_imp > 0) {
    const int n = 16 * ctx->n_imp;
    int *sl0, *sl1, *d_nr, *cnt;
    uint32_t *cd0;
    ICF_CUDA(ctx, cudaMallocAsync(&sl0, sizeof(int) * n, s));
    ICF_CUDA(ctx, cudaMallocAsync(&sl1, sizeof(int) * n, s));
    ICF_CUDA(ctx, cudaMallocAsync(&cd0, sizeof(uint32_t) * n, s));
    ICF_CUDA(ctx, cudaMallocAsync(&cnt, sizeof(int) * (n + 1), s));
    ICF_CUDA(ctx, cudaMallocAsync(&d_nr, sizeof(int), s));
    if (n + 2 > ctx->cr_cap || !ctx->d_cr) {
      cudaFree(ctx->d_cr);
      cudaFree(ctx->d_cr_slot);
      cudaFree(ctx->d_cr_off);
      cudaFree(ctx->d_cr_range);
      cudaFree(ctx->d_cr_pslot);
      cudaFree(ctx->d_cr_row);
      ctx->d_cr = nullptr;
      ctx->d_cr_slot = ctx->d_cr_off = nullptr;
      ctx->d_cr_range = nullptr;
      ctx->d_cr_pslot = ctx->d_cr_row = nullptr;
      const long long cap = 2LL * n + 2;
      ICF_CUDA(ctx, cudaMalloc(&ctx->d_cr, sizeof(uint32_t) * (size_t)cap));
      ICF_CUDA(ctx, cudaMalloc(&ctx->d_cr_slot, sizeof(int) * (size_t)cap));
      ICF_CUDA(ctx, cudaMalloc(&ctx->d_cr_off, sizeof(int) * (size_t)cap));
      ICF_CUDA(ctx, cudaMalloc(&ctx->d_cr_range, sizeof(int2) * (size_t)cap));
      ICF_CUDA(ctx, cudaMalloc(&ctx->d_cr_pslot, sizeof(int) * (size_t)cap));
      ICF_CUDA(ctx, cudaMalloc(&ctx->d_cr_row, sizeof(int) * (size_t)cap));
      ctx->cr_cap = (int)cap;
    }
    k_cand_imp_rc<<<icf_blocks(ctx->n_imp, 128), 128, 0, s>>>(ctx->n_imp, ctx->d_imp, ctx->d_alt,
                                                             ctx->d_mkeys, nnz, sl0, cd0);
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, sl0, sl1, cd0, ctx->d_cr, n, 0, 32, s);
    if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
    ICF_CUDA(ctx, cub::DeviceRadixSort::SortPairs(ctx->d_tmp, tb, sl0, sl1, cd0, ctx->d_cr, n, 0, 32, s));
    tb = 0;
    cub::DeviceRunLengthEncode::Encode(nullptr, tb, sl1, ctx->d_cr_slot, cnt, d_nr, n, s);
    if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
    ICF_CUDA(ctx, cub::DeviceRunLengthEncode::Encode(ctx->d_tmp, tb, sl1, ctx->d_cr_slot, cnt, d_nr, n, s));
    int nr = 0;
    ICF_CUDA(ctx, cudaMemcpyAsync(&nr, d_nr, sizeof(int), cudaMemcpyDeviceToHost, s));
    ICF_CUDA(ctx, cudaStreamSynchronize(s));
    // the last run is the invalid slot marker when any candidate was skipped
    int last = 0;
    if (nr > 0) {
      ICF_CUDA(ctx, cudaMemcpyAsync(&last, ctx->d_cr_slot + nr - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
      ICF_CUDA(ctx, cudaStreamSynchronize(s));
    }
    const int nvalid = (nr > 0 && last == 0x7fffffff) ? nr - 1 : nr;
    ICF_CUDA(ctx, cudaMemsetAsync(cnt + nr, 0, sizeof(int), s));
    tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, ctx->d_cr_off, nr + 1, s);
    if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
    ICF_CUDA(ctx, cub::DeviceScan::ExclusiveSum(ctx->d_tmp, tb, cnt, ctx->d_cr_off, nr + 1, s));
    ICF_CUDA(ctx, cudaFreeAsync(sl0, s));
    ICF_CUDA(ctx, cudaFreeAsync(sl1, s));
    ICF_CUDA(ctx, cudaFreeAsync(cd0, s));
    ICF_CUDA(ctx, cudaFreeAsync(cnt, s));
    ICF_CUDA(ctx, cudaFreeAsync(d_nr, s));
    ctx->n_crs = nvalid;
    // where each code's record goes (k_imp_deriv writes, k_imp_add reads)
    if (n > ctx->imp_pos_cap || !ctx->d_imp_pos) {
      cudaFree(ctx->d_imp_pos);
      ctx->d_imp_pos = nullptr;
      ICF_CUDA(ctx, cudaMalloc(&ctx->d_imp_pos, sizeof(int) * 2 * (size_t)n));
      ctx->imp_pos_cap = 2LL * n;
    }
    ICF_CUDA(ctx, cudaMemsetAsync(ctx->d_imp_pos, 0xFF, sizeof(int) * (size_t)n, s));
    k_imp_pos<<<icf_blocks(n, 256), 256, 0, s>>>(n, ctx->d_cr_off + nvalid, ctx->d_cr, ctx->d_imp_pos);
    ICF_CUDA(ctx, cudaGetLastError());
    // how many of them the off-diagonal gather writes, and the launch order
    ctx->n_crs_off = 0;
    if (nvalid > 0) {
      int *d_flag, *d_pref;
      ICF_CUDA(ctx, cudaMallocAsync(&d_flag, sizeof(int) * (nvalid + 1LL), s));
      ICF_CUDA(ctx, cudaMallocAsync(&d_pref, sizeof(int) * (nvalid + 1LL), s));
      k_flag_off<<<icf_blocks(nvalid + 1LL, 256), 256, 0, s>>>(nvalid, ctx->d_cr_slot, ctx->d_mkeys, ctx->d_src,
                                                              ctx->src_identity ? 1 : 0, d_flag);
      tb = 0;
      cub::DeviceScan::ExclusiveSum(nullptr, tb, d_flag, d_pref, nvalid + 1, s);
      if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
      ICF_CUDA(ctx, cub::DeviceScan::ExclusiveSum(ctx->d_tmp, tb, d_flag, d_pref, nvalid + 1, s));
      ICF_CUDA(ctx, cudaMemcpyAsync(&ctx->n_crs_off, d_pref + nvalid, sizeof(int), cudaMemcpyDeviceToHost, s));
      ICF_CUDA(ctx, cudaStreamSynchronize(s));
      k_split_off<<<icf_blocks(nvalid, 256), 256, 0, s>>>(nvalid, nvalid - ctx->n_crs_off, ctx->d_cr_slot,
                                                           ctx->d_cr_off, ctx->d_mkeys, d_pref, ctx->d_cr_range,
                                                           ctx->d_cr_pslot, ctx->d_cr_row);
      ICF_CUDA(ctx, cudaGetLastError());
      ICF_CUDA(ctx, cudaFreeAsync(d_flag, s));
      ICF_CUDA(ctx, cudaFreeAsync(d_pref, s));
    }
    // impact staging
    if (ctx->n_imp > ctx->ks_cap) {
      cudaFree(ctx->d_ks);
      ctx->d_ks = nullptr;
      const size_t cap = 2 * (size_t)ctx->n_imp;
      ICF_CUDA(ctx, cudaMalloc(&ctx->d_ks, sizeof(double) * ICF_IMP_STAGE * cap));
      ctx->ks_cap = (int)cap;
    }
  }
  // outputs
  if ((long long)nnz * 9 > ctx->vals_cap || !ctx->d_vals) {
    cudaFree(ctx->d_vals);
    ctx->d_vals = nullptr;
    const long long c = 9LL * (nnz + nnz / 8 + 64);
    ICF_CUDA(ctx, cudaMalloc(&ctx->d_vals, sizeof(double) * (size_t)c));
    ctx->vals_cap = (int)(c > 0x7fffffff ? 0x7fffffff : c);
  }
  cudaFree(ctx->d_rhs);
  ctx->d_rhs = nullptr;
  ICF_CUDA(ctx, cudaMalloc(&ctx->d_rhs, sizeof(double) * (size_t)(3LL * N + 3)));
  ICF_CUDA(ctx, cudaStreamSynchronize(s));
  return ICF_OK;
}

int icf_launch_pcsr(icf_ctx *ctx, int kind, int *d_out) {
  cudaStream_t s = ctx->stream;
  if (kind == 0 && ctx->n_elem)
    k_pcsr<<<icf_blocks(ctx->n_elem, 128), 128, 0, s>>>(ctx->n_elem, 4, reinterpret_cast<const int *>(ctx->d_elem),
                                                       4, ctx->d_alt, ctx->d_mkeys, ctx->nnz, d_out);
  else if (kind == 1 && ctx->n_cz)
    k_pcsr<<<icf_blocks(ctx->n_cz, 128), 128, 0, s>>>(ctx->n_cz, 6, ctx->d_cz, 8, ctx->d_alt, ctx->d_mkeys,
                                                     ctx->nnz, d_out);
  else if (kind == 2 && ctx->n_imp)
    k_pcsr<<<icf_blocks(ctx->n_imp, 128), 128, 0, s>>>(ctx->n_imp, 4, reinterpret_cast<const int *>(ctx->d_imp),
                                                      4, ctx->d_alt, ctx->d_mkeys, ctx->nnz, d_out);
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}

__global__ void k_remap_units(long long n, const int2 *__restrict__ us, const int *__restrict__ s2m, int identity,
                              int2 *__restrict__ u) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int2 v = us[i];
  if (v.x >= 0 && !identity) v.x = s2m[v.x];
  u[i] = v;
}

int icf_remap_lists(icf_ctx *ctx) {
  const int ident = (ctx->src_identity || !ctx->d_s2m) ? 1 : 0;
  for (icf_sell *L : {&ctx->sell_off, &ctx->sell_diag, &ctx->sell_off_cz, &ctx->sell_diag_cz}) {
    if (L->n_slices == 0) continue;
    const long long n = (long long)(32 / L->lanes) * L->n_slices;  // units per slice: 32 / lanes
    k_remap_units<<<icf_blocks(n, 256), 256, 0, ctx->stream>>>(n, L->unit_s, ctx->d_s2m, ident, L->unit);
  }
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}

int icf_rebuild_lists(icf_ctx *ctx) {
  if (!ctx->have_structure) return icf_fail(ctx, ICF_ERR_STATE, "icf_create_structure first");
  if (build_lists(ctx, true, true)) return ICF_ERR_CUDA;
  if (icf_build_contrib(ctx)) return ICF_ERR_CUDA;
  if (icf_remap_lists(ctx)) return ICF_ERR_CUDA;
  ctx->version++;
  return ICF_OK;
}

int icf_rebuild_sell_diag(icf_ctx *ctx, int lanes) {
  if (!ctx->have_structure) return icf_fail(ctx, ICF_ERR_STATE, "icf_create_structure first");
  ctx->sell_diag.lanes = ctx->sell_diag_cz.lanes = lanes;
  if (build_lists(ctx, false, true)) return ICF_ERR_CUDA;
  if (icf_build_contrib(ctx)) return ICF_ERR_CUDA;
  if (icf_remap_lists(ctx)) return ICF_ERR_CUDA;
  ICF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return ICF_OK;
}

int icf_rebuild_sell_off(icf_ctx *ctx, bool natural) {
  if (!ctx->have_structure) return icf_fail(ctx, ICF_ERR_STATE, "icf_create_structure first");
  ctx->sell_off.natural = ctx->sell_off_cz.natural = natural;
  if (build_lists(ctx, true, false)) return ICF_ERR_CUDA;
  if (icf_build_contrib(ctx)) return ICF_ERR_CUDA;
  if (icf_remap_lists(ctx)) return ICF_ERR_CUDA;
  ICF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return ICF_OK;
}

// tetpos[16 e + 4 a + b] = position of tet code (e, a, b) in a gather list
__global__ void k_tetpos(long long n, const uint32_t *__restrict__ codes, int *__restrict__ tetpos) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const uint32_t c = codes[p];
  if (c == ICF_CODE_PAD || (c >> 30) != ICF_KIND_TET) return;
  const uint32_t e = (c >> 4) & 0x3FFFFFFu, a = (c >> 2) & 3u, b = c & 3u;
  tetpos[16 * (size_t)e + 4 * a + b] = (int)p;
}

int icf_build_contrib(icf_ctx *ctx) {
  cudaStream_t s = ctx->stream;
  const long long ne = ctx->n_elem;
  // only the contribution layout needs the map and its staging
  if (ne == 0 || ctx->layout != ICF_LAYOUT_CONTRIB) return ICF_OK;
  if (16 * ne > ctx->tetpos_cap || !ctx->d_tetpos) {
    cudaFree(ctx->d_tetpos);
    ctx->d_tetpos = nullptr;
    ICF_CUDA(ctx, cudaMalloc(&ctx->d_tetpos, sizeof(int) * 16 * (size_t)ne));
    ctx->tetpos_cap = 16 * ne;
  }
  ICF_CUDA(ctx, cudaMemsetAsync(ctx->d_tetpos, 0xff, sizeof(int) * 16 * (size_t)ne, s));
  const icf_sell *L[2] = {&ctx->sell_off, &ctx->sell_diag};
  void **stage[2] = {&ctx->d_stage_off, &ctx->d_stage_diag};
  long long *cap[2] = {&ctx->stage_off_cap, &ctx->stage_diag_cap};
  for (int k = 0; k < 2; k++) {
    const long long n = L[k]->n_codes;
    const long long bytes = (n > 0 ? n : 1) * (long long)ICF_CONTRIB_BYTES;
    if (bytes > *cap[k] || !*stage[k]) {
      cudaFree(*stage[k]);
      *stage[k] = nullptr;
      const long long c = bytes + bytes / 4;
      ICF_CUDA(ctx, cudaMalloc(stage[k], (size_t)c));
      *cap[k] = c;
    }
    // positions no tet writes (padding, CZ iterations) must read as zero
    ICF_CUDA(ctx, cudaMemsetAsync(*stage[k], 0, (size_t)bytes, s));
    if (n > 0) k_tetpos<<<icf_blocks(n, 256), 256, 0, s>>>(n, L[k]->codes, ctx->d_tetpos);
  }
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}
