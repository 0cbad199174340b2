// icf_broad.cu -- broad phase on the device: candidate surface-element pairs.
//
// The reference builds a k-DOP-24 bounding-volume tree on the host every few
// steps, refits it otherwise and self-collides it to list the element pairs
// its narrow phase tests (BVHT.cs:29-77, BVHN.cs:39-194, kDOP24.cs:69-169).
// Only that pair list crosses into the assembly path.  Here it is built where
// the positions already are, with a uniform grid:
//   1. axis-aligned box of every surface element at the current positions
//      (x0 + un), widened by `pad`;
//   2. cell size = the mean box extent (at least a sixteenth of the largest);
//      every (cell, element) entry of every cell a box reaches is listed and
//      the entries are sorted by cell (CUB radix sort);
//   3. within each cell, every pair a < b of elements whose boxes overlap
//      (closed intervals), that share no node and where a vertex of one lies
//      in the other's box is a candidate (with groups set, only pairs of
//      different groups);
//   4. a pair is reported only in the cell that holds the low corner of the
//      two boxes' intersection (so once), the pairs are sorted (a, b)
//      ascending, and the list stays on the device for the narrow phase.
// The pair set does not depend on the cell size: two overlapping boxes
// share the cell of their intersection's low corner; the host pair rule the
// tests compare against (a grid of its own) gives the same set.
// Like the reference's BVH, which holds every surface element of every mesh,
// pairs of one mesh are candidates: across a grain boundary the split node
// copies let two grains of one mesh interpenetrate, and the narrow phase turns
// that into impacts.  Optional groups (icf_set_surface_groups) restrict the
// pairs to different groups.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "icf_collide.cuh"
#include "icf_internal.cuh"

namespace {

struct box {
  double lo[3], hi[3];
};

__device__ __forceinline__ box elem_box(const int4 *selem, const double4 *xc, int i, double pad) {
  const int4 id = selem[i];
  const int n[4] = {id.x, id.y, id.z, id.w};
  box b;
  for (int k = 0; k < 3; k++) {
    b.lo[k] = 1e300;
    b.hi[k] = -1e300;
  }
  for (int v = 0; v < 4; v++) {
    const double4 p = xc[n[v]];
    const double c[3] = {p.x, p.y, p.z};
    for (int k = 0; k < 3; k++) {
      b.lo[k] = fmin(b.lo[k], c[k]);
      b.hi[k] = fmax(b.hi[k], c[k]);
    }
  }
  for (int k = 0; k < 3; k++) {
    b.lo[k] -= pad;
    b.hi[k] += pad;
  }
  return b;
}

__global__ void k_boxes(int n, const int4 *__restrict__ selem, const double4 *__restrict__ xc, double pad,
                        double *__restrict__ lohi, double *__restrict__ ext) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0;
  if (i < n) {
    const box b = elem_box(selem, xc, i, pad);
    for (int k = 0; k < 3; k++) {
      lohi[6 * (size_t)i + k] = b.lo[k];
      lohi[6 * (size_t)i + 3 + k] = b.hi[k];
      e = fmax(e, b.hi[k] - b.lo[k]);
    }
  }
  if (i < n) ext[i] = e;
}

// per element: its lowest cell and how many more it spans along each axis
// (every cell its box reaches; at most 16 more, the cell size being at least
// a sixteenth of the largest box): clo = {c0x, c0y, c0z, sx | sy << 10 | sz << 20}
__device__ __forceinline__ int cell_of(double v, double base, double cell) { return (int)floor((v - base) / cell); }
__global__ void k_cells(int n, const double *__restrict__ lohi, const double *__restrict__ red, int *__restrict__ cnt,
                        int4 *__restrict__ clo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double cell = red[0];
  int c0[3], sp[3];
  for (int k = 0; k < 3; k++) {
    c0[k] = cell_of(lohi[6 * (size_t)i + k], red[1 + k], cell);
    const int c1 = cell_of(lohi[6 * (size_t)i + 3 + k], red[1 + k], cell);
    sp[k] = c1 - c0[k];
  }
  cnt[i] = (sp[0] + 1) * (sp[1] + 1) * (sp[2] + 1);
  clo[i] = make_int4(c0[0], c0[1], c0[2], sp[0] | sp[1] << 10 | sp[2] << 20);
}


// With groups packed into the key (gbits >= 0), an entry's key is
// (x << 2 nb | y << nb | z) << gbits | group: sorted, the entries of a cell
// come in runs of one group each.
__global__ void k_entries(int n, const int4 *__restrict__ clo, const int *__restrict__ off, int nb, int gbits,
                          const int *__restrict__ group, unsigned long long *__restrict__ key,
                          int *__restrict__ elem) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int4 c = clo[i];
  int o = off[i];
  const unsigned long long g = gbits >= 0 ? (unsigned long long)(unsigned)group[i] : 0ull;
  const int sx = c.w & 1023, sy = (c.w >> 10) & 1023, sz = (c.w >> 20) & 1023;
  for (int dz = 0; dz <= sz; dz++)
    for (int dy = 0; dy <= sy; dy++)
      for (int dx = 0; dx <= sx; dx++) {
        // (x << 2 nb | y << nb | z) << gbits | group, or without groups the
        // cell alone (gbits < 0)
        const unsigned long long ck = ((unsigned long long)(unsigned)(c.x + dx) << (2 * nb)) |
                                      ((unsigned long long)(unsigned)(c.y + dy) << nb) |
                                      (unsigned long long)(unsigned)(c.z + dz);
        key[o] = gbits >= 0 ? (ck << gbits) | g : ck;
        elem[o] = i;
        o++;
      }
}

// first index in [lo, hi) whose key is > v
__device__ __forceinline__ int upper_key(const unsigned long long *key, int lo, int hi, unsigned long long v) {
  while (lo < hi) {
    const int mid = lo + ((hi - lo) >> 1);
    if (key[mid] <= v) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// vertex_in_box and keep_pair (the pair rule): icf_collide.cuh

// entry i pairs with the later entries of its cell; count, then write.  With
// group keys (gbits >= 0) the later entries of its own group are skipped: the
// candidates are the entries from the end of its (cell, group) run to the end
// of its cell, found by binary search.
__global__ void k_pairs(int m, const unsigned long long *__restrict__ key, const int *__restrict__ elem,
                        const double *__restrict__ lohi, const int4 *__restrict__ clo, int nb,
                        const int *__restrict__ group, int gbits,
                        const int4 *__restrict__ selem, const double4 *__restrict__ xc, const int *__restrict__ off,
                        int *__restrict__ cnt, unsigned long long *__restrict__ out, long long cap, int pb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const unsigned long long here = key[i];
  const int a0 = elem[i];
  int c = 0;
  int o = off ? off[i] : 0;
  int j0 = i + 1, j1 = m;
  if (gbits >= 0) {
    j0 = upper_key(key, i + 1, m, here);  // end of the run of this cell and group
    j1 = upper_key(key, j0, m, here | ((1ull << gbits) - 1));  // end of the cell
  }
  // this entry's cell, to report a pair only in the cell that holds the low
  // corner of the two boxes' intersection (each pair once)
  const unsigned long long ck = gbits >= 0 ? here >> gbits : here, mk = (1ull << nb) - 1;
  const int cx = (int)(ck >> (2 * nb)), cy = (int)((ck >> nb) & mk), cz = (int)(ck & mk);
  for (int j = j0; j < j1 && (gbits >= 0 || key[j] == here); j++) {
    const int b0 = elem[j];
    const int a = a0 < b0 ? a0 : b0, b = a0 < b0 ? b0 : a0;
    // the cell index is monotone in the coordinate, so the cell of the
    // intersection's low corner is the larger of the two low cells
    const int4 ca = clo[a], cb = clo[b];
    if (max(ca.x, cb.x) != cx || max(ca.y, cb.y) != cy || max(ca.z, cb.z) != cz) continue;
    if (keep_pair(a, b, lohi, group, selem, xc)) {
      // beyond the capacity nothing is written; the host sees the total
      // and repeats with a larger buffer
      if (out && o < cap) out[o] = ((unsigned long long)(unsigned)a << pb) | (unsigned)b;
      o++;
      c++;
    }
  }
  if (cnt) cnt[i] = c;
}

// The sorted pairs in[0 .. *n_all) (each reported once; the all-ones padding
// sorts after them) into the pair list; n_out[0] = the pair count.
__global__ void k_unpack_pairs(long long cap, const int *__restrict__ n_all, int *__restrict__ n_out,
                               const unsigned long long *__restrict__ in, int pb, int *__restrict__ pairs) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = *n_all < cap ? *n_all : cap;
  if (i == 0) *n_out = (int)n;
  if (i >= n) return;
  pairs[2 * (size_t)i] = (int)(in[i] >> pb);
  pairs[2 * (size_t)i + 1] = (int)(in[i] & ((1ull << pb) - 1));
}



// The grid: v[0] = largest extent, v[1..3] = lowest corner, v[4..6] = highest
// corner, v[7] = sum of extents, per block then one block over the partials
// (min and max are exact; the sum's order is fixed by the launch); the final
// block turns v[0] into the cell size, the mean extent but at least a
// sixteenth of the largest one, so that a box spans at most 17 cells per axis.
__device__ __forceinline__ void red8_block(double v[8]) {
  __shared__ double sh[8][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 8; q++) {
    const bool mn = q >= 1 && q <= 3, sum = q == 7;
    for (int o = 16; o > 0; o >>= 1) {
      const double t = __shfl_xor_sync(0xffffffffu, v[q], o);
      v[q] = sum ? v[q] + t : (mn ? fmin(v[q], t) : fmax(v[q], t));
    }
    if (lane == 0) sh[q][w] = v[q];
  }
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const bool mn = q >= 1 && q <= 3, sum = q == 7;
      v[q] = lane < nw ? sh[q][lane] : (sum ? 0.0 : (mn ? 1e300 : -1e300));
      for (int o = 16; o > 0; o >>= 1) {
        const double t = __shfl_xor_sync(0xffffffffu, v[q], o);
        v[q] = sum ? v[q] + t : (mn ? fmin(v[q], t) : fmax(v[q], t));
      }
    }
  }
}
__global__ void k_red7(int n, const double *__restrict__ lohi, const double *__restrict__ ext,
                       double *__restrict__ part) {
  double v[8] = {-1e300, 1e300, 1e300, 1e300, -1e300, -1e300, -1e300, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    v[0] = fmax(v[0], ext[i]);
    v[7] += ext[i];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      v[1 + k] = fmin(v[1 + k], lohi[6 * (size_t)i + k]);
      v[4 + k] = fmax(v[4 + k], lohi[6 * (size_t)i + 3 + k]);
    }
  }
  red8_block(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < 8; q++) part[8 * (size_t)blockIdx.x + q] = v[q];
}
__global__ void k_red7_final(int nb, int n, const double *__restrict__ part, double *__restrict__ red) {
  double v[8] = {-1e300, 1e300, 1e300, 1e300, -1e300, -1e300, -1e300, 0.0};
  for (int b = threadIdx.x; b < nb; b += blockDim.x)
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const bool mn = q >= 1 && q <= 3, sum = q == 7;
      const double x = part[8 * (size_t)b + q];
      v[q] = sum ? v[q] + x : (mn ? fmin(v[q], x) : fmax(v[q], x));
    }
  red8_block(v);
  if (threadIdx.x == 0) {
    const double mean = v[7] / n;
    v[0] = fmax(mean, v[0] / 16.0);
#pragma unroll
    for (int q = 0; q < 8; q++) red[q] = v[q];
  }
}

// ---- contact detection without the pair list ------------------------------------
// A pair (a, b) gives the impact (p, b) when p is a node of a, the narrow
// phase finds p strictly inside b, and (a, b) satisfies the pair rule.  So
// the impact list follows from one query per surface element b: the surface
// nodes p inside b's box (a grid of the surface nodes; b's box reaches every
// cell that can hold one), p not a node of b, p inside b (tet_contains with
// b's inverse, computed as k_narrow computes it, so the same bits), and some
// surface element a holding p with keep_pair(a, b).  Every (p, b) is found
// once (p lies in one cell).  tet_contains needs the barycentric coordinates
// above 1e-10, so such a p is strictly inside b's box.

__device__ __forceinline__ long long cell_lin(int x, int y, int z, int ny, int nz) {
  return ((long long)x * ny + y) * nz + z;
}

// count (off == nullptr) or place the surface nodes in the dense grid
// The detection grid's parameters, decided on the device: the cell (the mean
// box extent, at least a sixteenth of the largest) grows by 1.25 until the
// boxes' hull holds at most 8 n + 4096 cells.  gp = {nx, ny, nz, C, status}:
// status 0 ok, 1 degenerate boxes, 2 grid too large, 3 more cells than the
// buffers hold (cap cells + 1).
__global__ void k_grid_params(int n, long long cap, double *__restrict__ red, int *__restrict__ gp) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double cell = red[0];
  if (!(cell > 0) || !isfinite(cell)) {
    gp[4] = 1;
    return;
  }
  long long dims[3], C = 0;
  const long long lim = 8LL * n + 4096;
  for (int attempt = 0; attempt < 64; attempt++) {
    C = 1;
    for (int k = 0; k < 3; k++) {
      const double span = (red[4 + k] - red[1 + k]) / cell;
      dims[k] = (isfinite(span) && span < 1e12) ? (long long)span + 2 : (1LL << 40);
      C = (dims[k] > (1LL << 40) / (C > 1 ? C : 1)) ? (1LL << 40) : C * dims[k];
    }
    if (C <= lim) break;
    cell *= 1.25;
  }
  red[0] = cell;
  if (C > lim || dims[0] > INT32_MAX || dims[1] > INT32_MAX || dims[2] > INT32_MAX) {
    gp[4] = 2;
    return;
  }
  gp[0] = (int)dims[0];
  gp[1] = (int)dims[1];
  gp[2] = (int)dims[2];
  gp[3] = (int)C;
  gp[4] = (C + 1 > cap) ? 3 : 0;
}

// zero the first C + 1 counts of the grid's two counters (nothing when the
// parameters failed)
__global__ void k_grid_clear(const int *__restrict__ gp, int *__restrict__ a, int *__restrict__ b) {
  if (gp[4] != 0) return;
  const long long m = (long long)gp[3] + 1;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x) {
    a[i] = 0;
    b[i] = 0;
  }
}

// count (off == nullptr) or place the surface nodes in the dense grid
#define ICF_DET_IDBITS 26
__global__ void k_node_put(int ns, const int *__restrict__ snode, const double4 *__restrict__ xc,
                           const double *__restrict__ red, const int *__restrict__ gp, int *__restrict__ cnt,
                           const int *__restrict__ off, double4 *__restrict__ ent) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ns || gp[4] != 0) return;
  const int nx = gp[0], ny = gp[1], nz = gp[2];
  const double4 P = xc[snode[k]];
  const double cell = red[0];
  const int cx = cell_of(P.x, red[1], cell), cy = cell_of(P.y, red[2], cell), cz = cell_of(P.z, red[3], cell);
  // a node outside the grid is in no box (the grid spans every box)
  if (cx < 0 || cy < 0 || cz < 0 || cx >= nx || cy >= ny || cz >= nz) return;
  const long long l = cell_lin(cx, cy, cz, ny, nz);
  const int w = atomicAdd(cnt + l, 1);
  // the fourth component carries the surface-node index and the node id,
  // k 2^26 + p (an integer below 2^52, exact in a double)
  if (off) ent[off[l] + w] = make_double4(P.x, P.y, P.z, (double)(((long long)k << ICF_DET_IDBITS) | snode[k]));
}

// per surface element, for the detection: its box (as k_boxes) and largest
// extent, and the inverse of its edge matrix (as k_narrow computes it) with
// its first vertex, 12 doubles; one read of its four nodes serves both
__global__ void k_boxes_inv(int n, const int4 *__restrict__ selem, const double4 *__restrict__ xc, double pad,
                            double *__restrict__ lohi, double *__restrict__ ext, double *__restrict__ inv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int4 id = selem[i];
  const int nn[4] = {id.x, id.y, id.z, id.w};
  double x[12];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const double4 p = xc[nn[k]];
    x[3 * k] = p.x; x[3 * k + 1] = p.y; x[3 * k + 2] = p.z;
  }
  double lo[3], hi[3], e = 0;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    lo[k] = fmin(fmin(fmin(x[k], x[3 + k]), x[6 + k]), x[9 + k]) - pad;
    hi[k] = fmax(fmax(fmax(x[k], x[3 + k]), x[6 + k]), x[9 + k]) + pad;
    e = fmax(e, hi[k] - lo[k]);
  }
  double2 *l = reinterpret_cast<double2 *>(lohi + 6 * (size_t)i);
  l[0] = make_double2(lo[0], lo[1]);
  l[1] = make_double2(lo[2], hi[0]);
  l[2] = make_double2(hi[1], hi[2]);
  ext[i] = e;
  double b[9];
  tet_inverse(x, b);
  double2 *o = reinterpret_cast<double2 *>(inv + 12 * (size_t)i);
  o[0] = make_double2(b[0], b[1]);
  o[1] = make_double2(b[2], b[3]);
  o[2] = make_double2(b[4], b[5]);
  o[3] = make_double2(b[6], b[7]);
  o[4] = make_double2(b[8], x[0]);
  o[5] = make_double2(x[1], x[2]);
}

// some surface element holding surface node k forms a candidate pair with b
// (only on a hit)
__device__ __forceinline__ bool pair_exists(int k, int b, const int *__restrict__ sinc_off, const int *__restrict__ sinc,
                                         const double *__restrict__ lohi, const int *__restrict__ group,
                                         const int4 *__restrict__ selem, const double4 *__restrict__ xc) {
  for (int q = sinc_off[k]; q < sinc_off[k + 1]; q++) {
    const int a = sinc[q];
    if (keep_pair(a < b ? a : b, a < b ? b : a, lohi, group, selem, xc)) return true;
  }
  return false;
}

// DET_TPE threads per surface element b (four: 2, 8, 16 and 32 measured
// slower over cfg1 and cfg2): the entries of the cells its box reaches are
// dealt out by their index modulo DET_TPE, so the threads share the work
// evenly however it falls into cells; keys k << eb | b of the surface nodes k
// strictly inside b (candidates for k_pair_check)
#ifndef DET_MINB
#define DET_MINB 8
#endif
#ifndef DET_TPE
#define DET_TPE 4  // threads per surface element (a power of two)
#endif
__global__ void __launch_bounds__(128, DET_MINB) k_detect(int n, const int4 *__restrict__ selem, const double4 *__restrict__ xc,
                                                const double *__restrict__ lohi, const int4 *__restrict__ clo,
                                                const int *__restrict__ gp, const int *__restrict__ goff,
                                                const double4 *__restrict__ gnode, int eb,
                                                unsigned long long *__restrict__ out, long long cap,
                                                int *__restrict__ count, const double *__restrict__ inv) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int b = (int)(t / DET_TPE), g = (int)(t % DET_TPE);
  if (b >= n || gp[4] != 0) return;
  const int ny = gp[1], nz = gp[2];
  const int4 B = selem[b];
  const double *lh = lohi + 6 * (size_t)b;
  const double lx = lh[0], ly = lh[1], lz = lh[2], hx = lh[3], hy = lh[4], hz = lh[5];
  const int4 c = clo[b];
  const int sx = c.w & 1023, sy = (c.w >> 10) & 1023, sz = (c.w >> 20) & 1023;
  // the (x, y) columns of the box's cells: a run of cells along z is
  // contiguous in the grid, so a column's entries are one range; the next
  // column's range is read while this one's entries are tested
  const int ncol = (sx + 1) * (sy + 1);
  long long l = cell_lin(c.x, c.y, c.z, ny, nz);
  int e0 = goff[l], e1 = goff[l + sz + 1];
  for (int j = 0; j < ncol; j++) {
    int f0 = 0, f1 = 0;
    if (j + 1 < ncol) {
      const int dx = (j + 1) / (sy + 1), dy = (j + 1) % (sy + 1);
      l = cell_lin(c.x + dx, c.y + dy, c.z, ny, nz);
      f0 = goff[l];
      f1 = goff[l + sz + 1];
    }
    // thread g takes the entries whose index is g modulo DET_TPE
    for (int e = e0 + ((g - e0) & (DET_TPE - 1)); e < e1; e += DET_TPE) {
      const double4 P = gnode[e];
      if (!(P.x >= lx && P.x <= hx && P.y >= ly && P.y <= hy && P.z >= lz && P.z <= hz)) continue;
      const long long kp = (long long)P.w;
      const int p = (int)(kp & ((1LL << ICF_DET_IDBITS) - 1));
      if (p == B.x || p == B.y || p == B.z || p == B.w) continue;
      // b's inverse and first vertex, read when a node lies in its box
      double bi[9], x0[3];
      {
        const double2 *r = reinterpret_cast<const double2 *>(inv + 12 * (size_t)b);
        const double2 r0 = r[0], r1 = r[1], r2 = r[2], r3 = r[3], r4 = r[4], r5 = r[5];
        bi[0] = r0.x; bi[1] = r0.y; bi[2] = r1.x; bi[3] = r1.y; bi[4] = r2.x; bi[5] = r2.y;
        bi[6] = r3.x; bi[7] = r3.y; bi[8] = r4.x;
        x0[0] = r4.y; x0[1] = r5.x; x0[2] = r5.y;
      }
      if (!tet_contains(bi, P.x - x0[0], P.y - x0[1], P.z - x0[2])) continue;
      // a candidate: the pair rule is checked by k_pair_check, one thread
      // per candidate, so that its chain of loads stalls no other entry
      const int k = (int)(kp >> ICF_DET_IDBITS);
      const int w = atomicAdd(count, 1);
      if (w < cap) out[w] = ((unsigned long long)(unsigned)k << eb) | (unsigned)b;
    }
    e0 = f0;
    e1 = f1;
  }
}

// the candidates k << eb | b that satisfy the pair rule (some surface element
// holding node k forms a candidate pair with b) are counted per surface node
// and in total; the others become ~0
__global__ void k_pair_check(long long cap, const int *__restrict__ count, unsigned long long *__restrict__ keys, int eb,
                             const int *__restrict__ sinc_off, const int *__restrict__ sinc,
                             const double *__restrict__ lohi, const int *__restrict__ group,
                             const int4 *__restrict__ selem, const double4 *__restrict__ xc, int *__restrict__ kcnt,
                             int *__restrict__ valid) {
  const long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= cap || h >= *count) return;
  const unsigned long long key = keys[h];
  const int k = (int)(key >> eb);
  const int b = (int)(key & ((1ull << eb) - 1));
  if (pair_exists(k, b, sinc_off, sinc, lohi, group, selem, xc)) {
    atomicAdd(kcnt + k, 1);
    atomicAdd(valid, 1);
  } else {
    keys[h] = ~0ull;
  }
}

// the hits grouped by surface node (ascending, so by node id): key
// node << eb | b at koff[k] + the node's running count
__global__ void k_place(long long cap, const int *__restrict__ count, const unsigned long long *__restrict__ in, int eb,
                        const int *__restrict__ koff, int *__restrict__ kcur, const int *__restrict__ snode,
                        unsigned long long *__restrict__ out) {
  const long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= cap || h >= *count) return;
  const unsigned long long key = in[h];
  if (key == ~0ull) return;  // failed the pair rule
  const int k = (int)(key >> eb);
  const unsigned long long b = key & ((1ull << eb) - 1);
  const long long p = (long long)koff[k] + atomicAdd(kcur + k, 1);
  if (p < cap) out[p] = ((unsigned long long)(unsigned)snode[k] << eb) | b;
}

// each surface node's few hits in ascending element order (insertion sort)
__global__ void k_sort_seg(int ns, long long cap, const int *__restrict__ koff, unsigned long long *__restrict__ keys) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ns) return;
  const int a = koff[k];
  const int e = (int)(koff[k + 1] < cap ? koff[k + 1] : cap);
  for (int i = a + 1; i < e; i++) {
    const unsigned long long v = keys[i];
    int j = i - 1;
    while (j >= a && keys[j] > v) {
      keys[j + 1] = keys[j];
      j--;
    }
    keys[j + 1] = v;
  }
}

}  // namespace

template <typename T>
static int grow(icf_ctx *ctx, T **p, long long n) {
  cudaFree(*p);
  *p = nullptr;
  ICF_CUDA(ctx, cudaMalloc(p, sizeof(T) * (size_t)(n > 0 ? n : 1)));
  return ICF_OK;
}

void icf_free_contact_ws(icf_ctx *ctx) {
  icf_contact_ws &W = ctx->cws;
  void *d[] = {W.lohi, W.ext, W.tmpv, W.red, W.bcnt, W.boff, W.clo, W.ek0, W.ek1, W.ee0, W.ee1, W.pc, W.po,
               W.p0, W.p1, W.ncnt, W.noff, W.nk0, W.nk1, W.d_small, W.gcnt, W.goff, W.gcur, W.gnode,
               W.kcnt, W.koff, W.kcur, W.tinv, W.gp};
  for (void *q : d) cudaFree(q);
  cudaFreeHost(W.h_small);
  cudaFreeHost(W.h_red);
  cudaFreeHost(W.h_gp);
  if (W.det_exec) cudaGraphExecDestroy(W.det_exec);
  W = icf_contact_ws();
}

static int ensure_small(icf_ctx *ctx) {
  icf_contact_ws &W = ctx->cws;
  if (!W.d_small) ICF_CUDA(ctx, cudaMalloc(&W.d_small, 8 * sizeof(int)));
  if (!W.h_small) ICF_CUDA(ctx, cudaMallocHost(&W.h_small, 8 * sizeof(int)));
  if (!W.h_red) ICF_CUDA(ctx, cudaMallocHost(&W.h_red, 8 * sizeof(double)));
  return ICF_OK;
}

// Two synchronisations: one for the grid (cell size and corners, which set
// the key layout) and the entry count, one for the result.  Buffers live in
// the context's workspace; only growth beyond the high-water mark allocates.
int icf_broad_phase_impl(icf_ctx *ctx, double pad, const int *d_group, int *n_pairs_out) {
  cudaStream_t s = ctx->stream;
  const int n = ctx->n_surf;
  icf_contact_ws &W = ctx->cws;
  *n_pairs_out = 0;
  ctx->n_pairs = 0;
  if (n < 2) return ICF_OK;
  ICF_TRY_RC(ensure_small(ctx));
  const int nbk = (int)std::min<long long>((n + 255) / 256, 2LL * ctx->n_sm);
  if (n > W.b_cap) {
    ICF_TRY_RC(grow(ctx, &W.lohi, 6LL * n));
    ICF_TRY_RC(grow(ctx, &W.ext, n));
    ICF_TRY_RC(grow(ctx, &W.bcnt, n + 1LL));
    ICF_TRY_RC(grow(ctx, &W.boff, n + 1LL));
    ICF_TRY_RC(grow(ctx, &W.clo, n));
    W.b_cap = n;
  }
  if (!W.tmpv) ICF_TRY_RC(grow(ctx, &W.tmpv, 8LL * (2 * ctx->n_sm + 1)));
  if (!W.red) ICF_TRY_RC(grow(ctx, &W.red, 8));
  k_boxes<<<icf_blocks(n, 256), 256, 0, s>>>(n, ctx->d_selem, ctx->d_xc, pad, W.lohi, W.ext);
  k_red7<<<nbk, 256, 0, s>>>(n, W.lohi, W.ext, W.tmpv);
  k_red7_final<<<1, 256, 0, s>>>(nbk, n, W.tmpv, W.red);
  k_cells<<<icf_blocks(n, 256), 256, 0, s>>>(n, W.lohi, W.red, W.bcnt, W.clo);
  ICF_CUDA(ctx, cudaMemsetAsync(W.bcnt + n, 0, sizeof(int), s));
  size_t tb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb, W.bcnt, W.boff, n + 1, s);
  if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
  ICF_CUDA(ctx, cub::DeviceScan::ExclusiveSum(ctx->d_tmp, tb, W.bcnt, W.boff, n + 1, s));
  ICF_CUDA(ctx, cudaMemcpyAsync(W.h_red, W.red, 7 * sizeof(double), cudaMemcpyDeviceToHost, s));
  ICF_CUDA(ctx, cudaMemcpyAsync(W.h_small + 3, W.boff + n, sizeof(int), cudaMemcpyDeviceToHost, s));
  ICF_CUDA(ctx, cudaStreamSynchronize(s));
  const double *h_red = W.h_red;
  if (!(h_red[0] > 0) || !std::isfinite(h_red[0])) return icf_fail(ctx, ICF_ERR_NUMERIC, "broad phase: degenerate boxes");
  const int m = W.h_small[3];
  // (cell, group) keys when the cell indices and group ids fit in 63 bits
  int nb = 1;
  {
    double span = 0;
    for (int k = 0; k < 3; k++) span = fmax(span, (h_red[4 + k] - h_red[1 + k]) / h_red[0]);
    const double cells = std::isfinite(span) ? span + 2.0 : 1e30;
    while (nb < 40 && (double)(1ull << nb) < cells) nb++;
  }
  if (3 * nb > 63) return icf_fail(ctx, ICF_ERR_SIZE, "broad phase: more grid cells than 63-bit keys hold");
  const int gbits = (d_group && ctx->sgroup_bits >= 0 && 3 * nb + ctx->sgroup_bits <= 63) ? ctx->sgroup_bits : -1;
  // pair keys a << pb | b over the bits of the element ids (the all-ones
  // padding sorts after every pair)
  int pb = 1;
  while ((1LL << pb) < (long long)n) pb++;
  if (m > W.ent_cap) {
    const long long c = m + m / 4 + 64;
    ICF_TRY_RC(grow(ctx, &W.ek0, c));
    ICF_TRY_RC(grow(ctx, &W.ek1, c));
    ICF_TRY_RC(grow(ctx, &W.ee0, c));
    ICF_TRY_RC(grow(ctx, &W.ee1, c));
    ICF_TRY_RC(grow(ctx, &W.pc, c + 1));
    ICF_TRY_RC(grow(ctx, &W.po, c + 1));
    W.ent_cap = c;
  }
  k_entries<<<icf_blocks(n, 256), 256, 0, s>>>(n, W.clo, W.boff, nb, gbits, d_group, W.ek0, W.ee0);
  const int end_bit = gbits >= 0 ? 3 * nb + gbits : 3 * nb;
  tb = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, W.ek0, W.ek1, W.ee0, W.ee1, m, 0, end_bit, s);
  if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
  ICF_CUDA(ctx, cub::DeviceRadixSort::SortPairs(ctx->d_tmp, tb, W.ek0, W.ek1, W.ee0, W.ee1, m, 0, end_bit, s));
  k_pairs<<<icf_blocks(m, 128), 128, 0, s>>>(m, W.ek1, W.ee1, W.lohi, W.clo, nb, d_group, gbits, ctx->d_selem, ctx->d_xc,
                                              nullptr, W.pc, nullptr, 0, 0);
  ICF_CUDA(ctx, cudaMemsetAsync(W.pc + m, 0, sizeof(int), s));
  tb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb, W.pc, W.po, m + 1, s);
  if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
  ICF_CUDA(ctx, cub::DeviceScan::ExclusiveSum(ctx->d_tmp, tb, W.pc, W.po, m + 1, s));
  for (int attempt = 0; attempt < 2; attempt++) {
    if (W.pair_cap == 0) {
      const long long c = std::max<long long>(4LL * n, 1024);
      ICF_TRY_RC(grow(ctx, &W.p0, c));
      ICF_TRY_RC(grow(ctx, &W.p1, c));
      W.pair_cap = c;
    }
    const long long P = W.pair_cap;
    if (P > ctx->pairs_cap || !ctx->d_pairs) {
      cudaFree(ctx->d_pairs);
      cudaFree(ctx->d_masks);
      ctx->d_pairs = ctx->d_masks = nullptr;
      ICF_CUDA(ctx, cudaMalloc(&ctx->d_pairs, sizeof(int) * 2 * (size_t)P));
      ICF_CUDA(ctx, cudaMalloc(&ctx->d_masks, sizeof(int) * (size_t)P));
      ctx->pairs_cap = (int)P;
    }
    // pad with all-ones keys: they sort after every pair and form one run
    ICF_CUDA(ctx, cudaMemsetAsync(W.p0, 0xFF, sizeof(unsigned long long) * (size_t)P, s));
    k_pairs<<<icf_blocks(m, 128), 128, 0, s>>>(m, W.ek1, W.ee1, W.lohi, W.clo, nb, d_group, gbits, ctx->d_selem, ctx->d_xc,
                                                W.po, nullptr, W.p0, P, pb);
    tb = 0;
    // the padding is all ones in every bit, so sorting the low 2 pb bits
    // still puts it after the pairs
    cub::DeviceRadixSort::SortKeys(nullptr, tb, W.p0, W.p1, (int)P, 0, 2 * pb, s);
    if (icf_scratch(ctx, tb)) return ICF_ERR_CUDA;
    ICF_CUDA(ctx, cub::DeviceRadixSort::SortKeys(ctx->d_tmp, tb, W.p0, W.p1, (int)P, 0, 2 * pb, s));
    k_unpack_pairs<<<icf_blocks(P, 256), 256, 0, s>>>(P, W.po + m, W.d_small + 1, W.p1, pb, ctx->d_pairs);
    ICF_CUDA(ctx, cudaGetLastError());
    ICF_CUDA(ctx, cudaMemcpyAsync(W.h_small + 2, W.po + m, sizeof(int), cudaMemcpyDeviceToHost, s));
    ICF_CUDA(ctx, cudaMemcpyAsync(W.h_small + 1, W.d_small + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    ICF_CUDA(ctx, cudaStreamSynchronize(s));
    const long long nall = W.h_small[2];
    if (nall <= P) {
      ctx->n_pairs = W.h_small[1];
      *n_pairs_out = ctx->n_pairs;
      return ICF_OK;
    }
    // more candidate pairs than the buffer holds: grow it and write them again
    const long long c = nall + nall / 4 + 1024;
    ICF_TRY_RC(grow(ctx, &W.p0, c));
    ICF_TRY_RC(grow(ctx, &W.p1, c));
    W.pair_cap = c;
  }
  return icf_fail(ctx, ICF_ERR_SIZE, "broad phase: pair buffer growth did not converge");
}

// Contact detection without the pair list, one synchronisation: the grid's
// parameters are decided on the device (k_grid_params), and the buffers are
// sized by high-water marks.  When a call finds more cells or more hits than
// the buffers hold, its result is discarded, the buffers grow to what that
// call reported, and it runs again.
// The launches of one detection up to the sorted keys (no synchronisation),
// with the CUB scratch already sized.
static int enqueue_detect(icf_ctx *ctx, double pad, const int *d_group, int eb, cudaStream_t s) {
  const int n = ctx->n_surf, ns = ctx->n_snode;
  icf_contact_ws &W = ctx->cws;
  const int nbk = (int)std::min<long long>((n + 255) / 256, 2LL * ctx->n_sm);
  const long long cap_cells = W.cell_cap;
  k_boxes_inv<<<icf_blocks(n, 128), 128, 0, s>>>(n, ctx->d_selem, ctx->d_xc, pad, W.lohi, W.ext, W.tinv);
  k_red7<<<nbk, 256, 0, s>>>(n, W.lohi, W.ext, W.tmpv);
  k_red7_final<<<1, 256, 0, s>>>(nbk, n, W.tmpv, W.red);
  k_grid_params<<<1, 32, 0, s>>>(n, cap_cells, W.red, W.gp);
  // the surface nodes by cell (over the high-water count of cells: the
  // counts past this call's C are never read)
  k_grid_clear<<<2 * ctx->n_sm, 256, 0, s>>>(W.gp, W.gcnt, W.gcur);
  k_node_put<<<icf_blocks(ns, 256), 256, 0, s>>>(ns, ctx->d_snode, ctx->d_xc, W.red, W.gp, W.gcnt, nullptr, nullptr);
  size_t tb = ctx->tmp_bytes;
  ICF_CUDA(ctx, cub::DeviceScan::ExclusiveSum(ctx->d_tmp, tb, W.gcnt, W.goff, (int)cap_cells, s));
  k_node_put<<<icf_blocks(ns, 256), 256, 0, s>>>(ns, ctx->d_snode, ctx->d_xc, W.red, W.gp, W.gcur, W.goff, W.gnode);
  // every element's cells
  k_cells<<<icf_blocks(n, 256), 256, 0, s>>>(n, W.lohi, W.red, W.bcnt, W.clo);
  ICF_CUDA(ctx, cudaMemsetAsync(W.d_small + 5, 0, 2 * sizeof(int), s));
  ICF_CUDA(ctx, cudaMemsetAsync(W.kcnt, 0, sizeof(int) * (ns + 1LL), s));
  k_detect<<<icf_blocks((long long)DET_TPE * n, 128), 128, 0, s>>>(n, ctx->d_selem, ctx->d_xc, W.lohi, W.clo, W.gp, W.goff, W.gnode,
                                                   eb, W.nk0, W.nkey_cap, W.d_small + 5, W.tinv);
  k_pair_check<<<icf_blocks(W.nkey_cap, 256), 256, 0, s>>>(W.nkey_cap, W.d_small + 5, W.nk0, eb, ctx->d_sinc_off,
                                                          ctx->d_sinc, W.lohi, d_group, ctx->d_selem, ctx->d_xc,
                                                          W.kcnt, W.d_small + 6);
  ICF_CUDA(ctx, cudaGetLastError());
  // grouped by surface node (a counting sort), each node's hits sorted: the
  // keys node << eb | element ascending
  tb = ctx->tmp_bytes;
  ICF_CUDA(ctx, cub::DeviceScan::ExclusiveSum(ctx->d_tmp, tb, W.kcnt, W.koff, ns + 1, s));
  ICF_CUDA(ctx, cudaMemsetAsync(W.kcur, 0, sizeof(int) * (ns + 1LL), s));
  k_place<<<icf_blocks(W.nkey_cap, 256), 256, 0, s>>>(W.nkey_cap, W.d_small + 5, W.nk0, eb, W.koff, W.kcur,
                                                     ctx->d_snode, W.nk1);
  k_sort_seg<<<icf_blocks(ns, 256), 256, 0, s>>>(ns, W.nkey_cap, W.koff, W.nk1);
  // the grid's status and size and the candidate count come back with the
  // impact count
  ICF_CUDA(ctx, cudaMemcpyAsync(W.h_gp, W.gp, 5 * sizeof(int), cudaMemcpyDeviceToHost, s));
  ICF_CUDA(ctx, cudaMemcpyAsync(W.h_small + 2, W.d_small + 5, sizeof(int), cudaMemcpyDeviceToHost, s));
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}

// Everything a captured detection depends on: replayed while these hold.
static void detect_key(const icf_ctx *ctx, double pad, const int *d_group, int eb, std::vector<long long> &k) {
  const icf_contact_ws &W = ctx->cws;
  long long pb;
  std::memcpy(&pb, &pad, sizeof(pb));
  k = {ctx->n_surf, ctx->n_snode, pb, eb, W.cell_cap, W.nkey_cap, (long long)ctx->tmp_bytes, ctx->n_sm,
       (long long)(intptr_t)d_group, (long long)(intptr_t)ctx->stream, (long long)(intptr_t)ctx->d_tmp,
       (long long)(intptr_t)ctx->d_selem, (long long)(intptr_t)ctx->d_xc, (long long)(intptr_t)ctx->d_snode,
       (long long)(intptr_t)ctx->d_sinc_off, (long long)(intptr_t)ctx->d_sinc, (long long)(intptr_t)W.lohi,
       (long long)(intptr_t)W.ext, (long long)(intptr_t)W.tmpv, (long long)(intptr_t)W.red,
       (long long)(intptr_t)W.gp, (long long)(intptr_t)W.h_gp, (long long)(intptr_t)W.tinv,
       (long long)(intptr_t)W.gcnt, (long long)(intptr_t)W.goff, (long long)(intptr_t)W.gcur,
       (long long)(intptr_t)W.gnode, (long long)(intptr_t)W.bcnt, (long long)(intptr_t)W.clo,
       (long long)(intptr_t)W.kcnt, (long long)(intptr_t)W.koff, (long long)(intptr_t)W.kcur,
       (long long)(intptr_t)W.nk0, (long long)(intptr_t)W.nk1, (long long)(intptr_t)W.d_small};
}

// One detection: the launches through a CUDA graph captured on first use and
// replayed while nothing it depends on changed, then the closest faces and
// the one synchronisation (icf_finish_impacts).
static int detect_pass(icf_ctx *ctx, double pad, const int *d_group, int *n_impacts, bool *again) {
  cudaStream_t s = ctx->stream;
  const int n = ctx->n_surf, ns = ctx->n_snode;
  icf_contact_ws &W = ctx->cws;
  *again = false;
  int eb = 1;
  while ((1LL << eb) < (long long)n) eb++;
  // the two scans' scratch, sized before any capture
  size_t tb1 = 0, tb2 = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb1, W.gcnt, W.goff, (int)W.cell_cap, s);
  cub::DeviceScan::ExclusiveSum(nullptr, tb2, W.kcnt, W.koff, ns + 1, s);
  if (icf_scratch(ctx, std::max(tb1, tb2))) return ICF_ERR_CUDA;
  std::vector<long long> key;
  detect_key(ctx, pad, d_group, eb, key);
  if (!W.det_exec || key != W.det_key) {
    if (W.det_exec) {
      cudaGraphExecDestroy(W.det_exec);
      W.det_exec = nullptr;
    }
    ICF_CUDA(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue_detect(ctx, pad, d_group, eb, s);
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(s, &g);
    if (rc != ICF_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (ec != cudaSuccess) return icf_fail(ctx, ICF_ERR_CUDA, std::string("detection capture: ") + cudaGetErrorString(ec));
    const cudaError_t ei = cudaGraphInstantiate(&W.det_exec, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
      W.det_exec = nullptr;
      return icf_fail(ctx, ICF_ERR_CUDA, std::string("detection graph: ") + cudaGetErrorString(ei));
    }
    W.det_key = key;
  }
  ICF_CUDA(ctx, cudaGraphLaunch(W.det_exec, s));
  ICF_TRY_RC(icf_finish_impacts(ctx, W.nk1, (int)W.nkey_cap, W.d_small + 6, eb, n_impacts));
  const int st = W.h_gp[4];
  if (st == 1) return icf_fail(ctx, ICF_ERR_NUMERIC, "contact detection: degenerate boxes");
  if (st == 2) return icf_fail(ctx, ICF_ERR_SIZE, "contact detection: grid too large");
  if (st == 3) {  // more cells than the buffers hold
    const long long c = W.h_gp[3] + W.h_gp[3] / 4 + 2;
    ICF_TRY_RC(grow(ctx, &W.gcnt, c));
    ICF_TRY_RC(grow(ctx, &W.goff, c));
    ICF_TRY_RC(grow(ctx, &W.gcur, c));
    ICF_CUDA(ctx, cudaMemsetAsync(W.gcnt, 0, sizeof(int) * (size_t)c, s));
    W.cell_cap = c;
    *again = true;
  }
  const long long hits = W.h_small[2];  // candidates, before the pair rule
  if (hits > W.nkey_cap) {  // more candidates than the key buffers hold
    const long long c = hits + hits / 4 + 1024;
    ICF_TRY_RC(grow(ctx, &W.nk0, c));
    ICF_TRY_RC(grow(ctx, &W.nk1, c));
    W.nkey_cap = c;
    *again = true;
  }
  return ICF_OK;
}

int icf_detect_contacts_impl(icf_ctx *ctx, double pad, const int *d_group, int *n_impacts) {
  const int n = ctx->n_surf, ns = ctx->n_snode;
  icf_contact_ws &W = ctx->cws;
  *n_impacts = 0;
  ctx->imp_cmp_valid = false;
  if (n < 2 || ns == 0) {
    ctx->n_imp = 0;
    return ICF_OK;
  }
  if (ctx->n_nodes >= (1 << ICF_DET_IDBITS) || ns >= (1 << ICF_DET_IDBITS))
    return icf_fail(ctx, ICF_ERR_SIZE, "contact detection: more than 2^26 nodes");
  ICF_TRY_RC(ensure_small(ctx));
  if (n > W.b_cap) {
    ICF_TRY_RC(grow(ctx, &W.lohi, 6LL * n));
    ICF_TRY_RC(grow(ctx, &W.ext, n));
    ICF_TRY_RC(grow(ctx, &W.bcnt, n + 1LL));
    ICF_TRY_RC(grow(ctx, &W.boff, n + 1LL));
    ICF_TRY_RC(grow(ctx, &W.clo, n));
    W.b_cap = n;
  }
  if (ns > W.gnode_cap) {
    ICF_TRY_RC(grow(ctx, &W.gnode, ns));
    W.gnode_cap = ns;
  }
  if (n > W.tinv_cap) {
    ICF_TRY_RC(grow(ctx, &W.tinv, 12LL * n));
    W.tinv_cap = n;
  }
  if (ns + 1LL > W.kcap) {
    ICF_TRY_RC(grow(ctx, &W.kcnt, ns + 1LL));
    ICF_TRY_RC(grow(ctx, &W.koff, ns + 1LL));
    ICF_TRY_RC(grow(ctx, &W.kcur, ns + 1LL));
    W.kcap = ns + 1LL;
  }
  if (!W.tmpv) ICF_TRY_RC(grow(ctx, &W.tmpv, 8LL * (2 * ctx->n_sm + 1)));
  if (!W.red) ICF_TRY_RC(grow(ctx, &W.red, 8));
  if (!W.gp) ICF_TRY_RC(grow(ctx, &W.gp, 8));
  if (!W.h_gp) ICF_CUDA(ctx, cudaMallocHost(&W.h_gp, 8 * sizeof(int)));
  if (W.cell_cap == 0) {  // a first guess: a cell per surface element
    const long long c = n + 4096LL;
    ICF_TRY_RC(grow(ctx, &W.gcnt, c));
    ICF_TRY_RC(grow(ctx, &W.goff, c));
    ICF_TRY_RC(grow(ctx, &W.gcur, c));
    // counts past a call's C are scanned but never read; start them at zero
    ICF_CUDA(ctx, cudaMemsetAsync(W.gcnt, 0, sizeof(int) * (size_t)c, ctx->stream));
    W.cell_cap = c;
  }
  if (W.nkey_cap == 0) {
    const long long c = std::max<long long>(n / 4, 1024);
    ICF_TRY_RC(grow(ctx, &W.nk0, c));
    ICF_TRY_RC(grow(ctx, &W.nk1, c));
    W.nkey_cap = c;
  }
  for (int attempt = 0; attempt < 3; attempt++) {
    bool again = false;
    ICF_TRY_RC(detect_pass(ctx, pad, d_group, n_impacts, &again));
    if (!again) return ICF_OK;
  }
  return icf_fail(ctx, ICF_ERR_SIZE, "contact detection: buffer growth did not converge");
}
