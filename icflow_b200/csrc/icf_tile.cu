// icf_tile.cu -- row tiles of the static pattern for the tiled gather.
//
// The list gathers (icf_gather.cu) read two staging records per contribution
// code straight from global memory: every code costs two scattered 32 B
// requests to L2, each behind the load of its code, and each tet's records
// are requested about ten times (six off-diagonal and four diagonal codes).
// The tiled gather instead gives one CTA a set of rows whose tets fit in
// shared memory: it copies each of those tets' four {h_a, V} records once
// (one line per tet) together with the tile's codes, then sums every block of
// its rows from shared memory.  A tet is copied once per tile that holds one
// of its vertices; cutting the rows in Morton order of their node positions
// keeps the tiles compact, so a tet lands in about two tiles.
//
// The tiles depend only on the static pattern (tets, CZs, rows), so they are
// built once, on the host, from the device pattern; each structure build only
// maps the static slots of the units to the merged ones (icf_remap_tiles).
// Each block is summed by one lane in the order of its codes in the static
// code list, as the off-diagonal list gather sums it.
#include <algorithm>
#include <cstdint>
#include <type_traits>
#include <vector>

#include "icf_internal.cuh"

namespace {

// 21-bit coordinate -> every third bit of a 63-bit Morton key
uint64_t spread3(uint32_t v) {
  uint64_t x = v & 0x1FFFFFu;
  x = (x | x << 32) & 0x001F00000000FFFFull;
  x = (x | x << 16) & 0x001F0000FF0000FFull;
  x = (x | x << 8) & 0x100F00F00F00F00Full;
  x = (x | x << 4) & 0x10C30C30C30C30C3ull;
  x = (x | x << 2) & 0x1249249249249249ull;
  return x;
}

__global__ void k_tile_units(long long n, const int2 *__restrict__ us, const int *__restrict__ s2m, int identity,
                             int2 *__restrict__ u) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int2 v = us[i];
  if (v.x >= 0 && !identity) v.x = s2m[v.x];
  u[i] = v;
}

struct unit_rec {
  int slot, row, nt, nc;
};

}  // namespace

void icf_free_tiles(icf_ctx *ctx) {
  icf_tiles &T = ctx->tiles;
  void *p[] = {T.tiles, T.trange, T.ttet, T.meta, T.unit_s, T.unit, T.tcodes, T.czcodes};
  for (void *q : p) cudaFree(q);
  T = icf_tiles();
}

bool icf_tiles_active(const icf_ctx *ctx) {
  return ctx->gather_tiles && ctx->tiles.built && ctx->tiles.ok && ctx->layout == ICF_LAYOUT_RECORDS &&
         ctx->tiles.n_tiles > 0;
}

int icf_build_tiles(icf_ctx *ctx) {
  icf_free_tiles(ctx);
  icf_tiles &T = ctx->tiles;
  T.built = true;
  const int N = ctx->N, nnz_s = ctx->nnz_s, ne = ctx->n_elem, nn = ctx->n_nodes;
  if (N == 0 || nnz_s == 0 || !ctx->d_skeys) return ICF_OK;
  // the static pattern and the node positions, on the host
  std::vector<unsigned long long> keys((size_t)nnz_s);
  std::vector<int> rc_off((size_t)nnz_s + 1), rc_mid((size_t)nnz_s), diag((size_t)N);
  std::vector<uint32_t> rc((size_t)ctx->n_rc);
  std::vector<double4> x0((size_t)nn);
  ICF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ICF_CUDA(ctx, cudaMemcpy(keys.data(), ctx->d_skeys, sizeof(unsigned long long) * keys.size(),
                           cudaMemcpyDeviceToHost));
  ICF_CUDA(ctx, cudaMemcpy(rc_off.data(), ctx->d_rc_off, sizeof(int) * rc_off.size(), cudaMemcpyDeviceToHost));
  ICF_CUDA(ctx, cudaMemcpy(rc_mid.data(), ctx->d_rc_mid, sizeof(int) * rc_mid.size(), cudaMemcpyDeviceToHost));
  ICF_CUDA(ctx, cudaMemcpy(diag.data(), ctx->d_diag, sizeof(int) * diag.size(), cudaMemcpyDeviceToHost));
  if (!rc.empty())
    ICF_CUDA(ctx, cudaMemcpy(rc.data(), ctx->d_rc, sizeof(uint32_t) * rc.size(), cudaMemcpyDeviceToHost));
  ICF_CUDA(ctx, cudaMemcpy(x0.data(), ctx->d_x0, sizeof(double4) * x0.size(), cudaMemcpyDeviceToHost));

  // slots of each row (the static keys are sorted by row, then column)
  std::vector<int> rp((size_t)N + 1, 0);
  for (int s = 0; s < nnz_s; s++) rp[(size_t)(keys[s] >> 32) + 1]++;
  for (int r = 0; r < N; r++) rp[r + 1] += rp[r];
  // rows in Morton order of their nodes
  std::vector<int> node_of((size_t)N, -1);
  for (int v = 0; v < nn && v < (int)ctx->h_alt.size(); v++) {
    const int r = ctx->h_alt[v];
    if (r >= 0 && r < N) node_of[r] = v;
  }
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int r = 0; r < N; r++) {
    if (node_of[r] < 0) continue;
    const double4 p = x0[node_of[r]];
    const double c[3] = {p.x, p.y, p.z};
    for (int k = 0; k < 3; k++) lo[k] = std::min(lo[k], c[k]), hi[k] = std::max(hi[k], c[k]);
  }
  double ext = 0;
  for (int k = 0; k < 3; k++) ext = std::max(ext, hi[k] - lo[k]);
  const double q = ext > 0 ? 2097151.0 / ext : 0.0;
  std::vector<std::pair<uint64_t, int>> ord((size_t)N);
  for (int r = 0; r < N; r++) {
    uint64_t key = 0;
    if (node_of[r] >= 0) {
      const double4 p = x0[node_of[r]];
      const double c[3] = {p.x, p.y, p.z};
      uint32_t b[3];
      for (int k = 0; k < 3; k++) {
        const double f = (c[k] - lo[k]) * q;
        b[k] = f <= 0 ? 0u : (f >= 2097151.0 ? 2097151u : (uint32_t)f);
      }
      key = spread3(b[0]) | spread3(b[1]) << 1 | spread3(b[2]) << 2;
    }
    ord[r] = {key, r};
  }
  std::sort(ord.begin(), ord.end());

  // greedy cut: a row joins the current tile while the tile's tets fit (and
  // while its tet codes stay within ICF_TILE_CODES).  The tets of a row are
  // those of its diagonal block's codes: every tet with a vertex on the row.
  auto tet_of = [](uint32_t code) { return (int)((code >> 4) & 0x3FFFFFFu); };
  std::vector<int> stamp((size_t)ne, -1);
  std::vector<int> bnd{0};
  int cur = 0, cur_tets = 0;
  long long cur_codes = 0;
  for (int i = 0; i < N; i++) {
    const int r = ord[i].second, s = diag[r];
    const int b0 = s >= 0 ? rc_off[s] : 0, b1 = s >= 0 ? rc_mid[s] : 0;
    if (b1 - b0 > ICF_TILE_TETS) return ICF_OK;  // T.ok stays false: the list gathers serve this model
    long long rcodes = 0;
    for (int sl = rp[r]; sl < rp[r + 1]; sl++) rcodes += rc_mid[sl] - rc_off[sl];
    int nw = 0;
    for (int k = b0; k < b1; k++) nw += stamp[tet_of(rc[k])] != cur;
    if (i > bnd.back() && (cur_tets + nw > ICF_TILE_TETS || cur_codes + rcodes > ICF_TILE_CODES)) {
      bnd.push_back(i);
      cur++;
      cur_tets = 0;
      cur_codes = 0;
      nw = b1 - b0;
    }
    for (int k = b0; k < b1; k++) stamp[tet_of(rc[k])] = cur;
    cur_tets += nw;
    cur_codes += rcodes;
  }
  bnd.push_back(N);
  const int nt_tiles = (int)bnd.size() - 1;

  // per tile: tets (ascending), units sorted by code counts, slices of 32
  std::vector<int4> h_tiles((size_t)nt_tiles);
  std::vector<int2> h_trange((size_t)nt_tiles);
  std::vector<int> h_ttet;
  std::vector<int4> h_meta;
  std::vector<int2> h_unit;
  std::vector<uint16_t> h_tcodes;
  std::vector<uint32_t> h_czcodes;
  std::vector<int> loc((size_t)ne, -1);
  std::fill(stamp.begin(), stamp.end(), -1);
  std::vector<int> tets;
  std::vector<unit_rec> units;
  long long n_real = 0, n_dg = 0, n_off = 0;
  size_t smem64 = 0, smem32 = 0, smemf64 = 0, smemf32 = 0;
  for (int t = 0; t < nt_tiles; t++) {
    tets.clear();
    units.clear();
    for (int i = bnd[t]; i < bnd[t + 1]; i++) {
      const int r = ord[i].second, s = diag[r];
      if (s >= 0)
        for (int k = rc_off[s]; k < rc_mid[s]; k++) {
          const int e = tet_of(rc[k]);
          if (stamp[e] != t) stamp[e] = t, tets.push_back(e);
        }
      for (int sl = rp[r]; sl < rp[r + 1]; sl++)
        units.push_back({sl, sl == s ? r : -1, rc_mid[sl] - rc_off[sl], rc_off[sl + 1] - rc_mid[sl]});
    }
    std::sort(tets.begin(), tets.end());
    for (int i = 0; i < (int)tets.size(); i++) loc[tets[i]] = i;
    std::stable_sort(units.begin(), units.end(), [](const unit_rec &a, const unit_rec &b) {
      return a.nt != b.nt ? a.nt > b.nt : a.nc > b.nc;
    });
    const int ns = ((int)units.size() + 31) / 32;
    const size_t t0 = h_tcodes.size();
    h_tiles[t] = make_int4((int)h_ttet.size(), (int)tets.size(), (int)h_meta.size(), ns);
    h_ttet.insert(h_ttet.end(), tets.begin(), tets.end());
    for (int sl = 0; sl < ns; sl++) {
      int mt = 0, mc = 0;
      const int u0 = 32 * sl, u1 = std::min((int)units.size(), u0 + 32);
      for (int u = u0; u < u1; u++) mt = std::max(mt, units[u].nt), mc = std::max(mc, units[u].nc);
      const size_t tb = h_tcodes.size(), cb = h_czcodes.size();
      h_meta.push_back(make_int4((int)tb, mt, mc, (int)cb));
      h_tcodes.resize(tb + 32 * (size_t)mt, (uint16_t)0xFFFFu);
      h_czcodes.resize(cb + 32 * (size_t)mc, ICF_CODE_PAD);
      for (int j = 0; j < 32; j++) {
        const int u = u0 + j;
        if (u >= u1) {
          h_unit.push_back(make_int2(-1, -1));
          continue;
        }
        const unit_rec &ur = units[u];
        h_unit.push_back(make_int2(ur.slot, ur.row));
        (ur.row >= 0 ? n_dg : n_off)++;
        n_real += ur.nt + ur.nc;
        for (int k = 0; k < ur.nt; k++) {
          const uint32_t c = rc[rc_off[ur.slot] + k];
          // every tet of a block has a vertex on the block's row, so it is
          // in the tile; anything else would index outside the staged records
          if (stamp[tet_of(c)] != t) return ICF_OK;  // T.ok stays false
          h_tcodes[tb + 32 * (size_t)k + j] = (uint16_t)(((uint32_t)loc[tet_of(c)] << 4) | (c & 15u));
        }
        for (int k = 0; k < ur.nc; k++) h_czcodes[cb + 32 * (size_t)k + j] = rc[rc_mid[ur.slot] + k];
      }
    }
    const size_t nc16 = h_tcodes.size() - t0;
    h_trange[t] = make_int2((int)t0, (int)nc16);
    // records, slice metadata, units, tet codes, tet ids
    const size_t rest = 16 * (size_t)ns + 256 * (size_t)ns + 2 * nc16 + 4 * tets.size();
    smem64 = std::max(smem64, 128 * tets.size() + rest);
    smem32 = std::max(smem32, 64 * tets.size() + rest);
    // fused: the records and 12 rhs values per tet, no tet ids
    smemf64 = std::max(smemf64, (128 + 96) * tets.size() + rest - 4 * tets.size());
    smemf32 = std::max(smemf32, (64 + 96) * tets.size() + rest - 4 * tets.size());
  }
  if (h_tcodes.size() >= (size_t)INT32_MAX || h_czcodes.size() >= (size_t)INT32_MAX || smem64 > 200 * 1024)
    return ICF_OK;  // offsets are 32-bit, shared memory bounded: the list gathers serve

  // upload
  auto up = [&](auto **d, const auto &h) -> int {
    typedef typename std::decay<decltype(h[0])>::type E;
    ICF_CUDA(ctx, cudaMalloc(d, sizeof(E) * std::max<size_t>(h.size(), 1)));
    if (!h.empty()) ICF_CUDA(ctx, cudaMemcpy(*d, h.data(), sizeof(E) * h.size(), cudaMemcpyHostToDevice));
    return ICF_OK;
  };
  ICF_TRY_RC(up(&T.tiles, h_tiles));
  ICF_TRY_RC(up(&T.trange, h_trange));
  ICF_TRY_RC(up(&T.ttet, h_ttet));
  ICF_TRY_RC(up(&T.meta, h_meta));
  ICF_TRY_RC(up(&T.unit_s, h_unit));
  ICF_TRY_RC(up(&T.tcodes, h_tcodes));
  ICF_TRY_RC(up(&T.czcodes, h_czcodes));
  ICF_CUDA(ctx, cudaMalloc(&T.unit, sizeof(int2) * std::max<size_t>(h_unit.size(), 1)));
  T.n_tiles = nt_tiles;
  T.n_slices = (int)h_meta.size();
  T.n_ttet = (long long)h_ttet.size();
  T.n_tcodes = (long long)h_tcodes.size();
  T.n_czcodes = (long long)h_czcodes.size();
  T.n_real = n_real;
  T.n_diag_units = n_dg;
  T.n_off_units = n_off;
  T.smem64 = smem64;
  T.smem32 = smem32;
  T.smemf64 = smemf64;
  T.smemf32 = smemf32;
  T.ok = true;
  ICF_TRY_RC(icf_gather_tile_setup(ctx));
  return icf_remap_tiles(ctx);
}

int icf_remap_tiles(icf_ctx *ctx) {
  icf_tiles &T = ctx->tiles;
  if (!T.built || !T.ok || T.n_slices == 0) return ICF_OK;
  const long long n = 32LL * T.n_slices;
  const int ident = (ctx->src_identity || !ctx->d_s2m) ? 1 : 0;
  k_tile_units<<<icf_blocks(n, 256), 256, 0, ctx->stream>>>(n, T.unit_s, ctx->d_s2m, ident, T.unit);
  ICF_CUDA(ctx, cudaGetLastError());
  return ICF_OK;
}
