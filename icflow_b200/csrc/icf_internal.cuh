// icf_internal.cuh -- shared definitions of the icflow_b200 library (not part
// of the public ABI).
//
// Device data layout (one context):
//   nodes     x0[n]  double4 {x, y, z, 0}        rest coordinates (static)
//             xc[n]  double4 {x, y, z, 0}        x0 + un of this iteration
//             va[n]  double2[3] {vx vy | vz ax | ay az}
//   tets      elem[ne] int4                       global node ids
//   CZs       cz[nc*8] int                        6 node ids + 2 pad (32 B)
//   CZ state  czs[nc*8] double                    pmax[3], tmax[3], pad
//   staging   es[ne*8] double4                    per tet vertex a:
//                                                 es[8e+a]   = {h_a, V}
//                                                 es[8e+4+a] = {rhs_a, 0}
//             cs[nc*48] double                    per CZ: 6 symmetric 3x3
//                                                 blocks Kt[i][j] (i<=j, 6 each)
//                                                 then rt[3][3], pad
//             ks[ni*132] double                   per impact: the records of its
//                                                 codes (<= 10 x 12) + 12 forces
//   pattern   static keys (row<<32|col) sorted, rc_off[nnz_s+1], rc[] codes
//             merged pattern rows/cols + src (static index of merged slot)
//
// Contribution codes (32 bit), one per (unit, row vertex a, column vertex b)
// with alt(b) >= alt(a):
//   bits 31..30 kind: 0 tet, 1 CZ, 2 impact
//   tet/impact: bits 29..4 unit, 3..2 a, 1..0 b
//   CZ:         bits 29..6 unit, 5..3 a, 2..0 b
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <functional>
#include <string>
#include <vector>

#include "../../include/icflow_b200.h"

#define ICF_KIND_TET 0u
#define ICF_KIND_CZ 1u
#define ICF_KIND_IMP 2u
#define ICF_MAX_TET_UNITS (1 << 26)
#define ICF_MAX_CZ_UNITS (1 << 24)
#define ICF_CZ_STAGE 48   // doubles per CZ in the staging buffer
#define ICF_IMP_STAGE 132 // doubles per impact in the staging buffer (allocation)
// The staging buffer of n impacts holds, from the start, one record of
// ICF_IMP_REC doubles per impact contribution code, at the code's position in
// the slot-sorted list d_cr (the 3x3 block of the code's vertex pair, then the
// rhs of the vertex on diagonal codes, else zeros; at most 10 codes per
// impact), and from ICF_IMP_FORCE_AT * n the 12 vertex forces of every impact.
#define ICF_IMP_REC 12
#define ICF_IMP_FORCE_AT 120
static_assert(ICF_IMP_FORCE_AT >= 10 * ICF_IMP_REC && ICF_IMP_STAGE >= ICF_IMP_FORCE_AT + 12,
              "impact staging: 10 code records, then 12 vertex forces");
__host__ __device__ inline double *icf_imp_forces(double *ks, long long n_imp) {
  return ks + (long long)ICF_IMP_FORCE_AT * n_imp;
}

// node -> (unit << 2 | vertex) incidence list in CSR form
struct icf_node_inc {
  int *off = nullptr, *inc = nullptr;
};

__host__ __device__ inline uint32_t icf_code_tet(uint32_t kind, uint32_t u,
                                                 uint32_t a, uint32_t b) {
  return (kind << 30) | (u << 4) | (a << 2) | b;
}
__host__ __device__ inline uint32_t icf_code_cz(uint32_t u, uint32_t a,
                                                uint32_t b) {
  return (ICF_KIND_CZ << 30) | (u << 6) | (a << 3) | b;
}

// Sliced-ELL contribution lists of a gather.  The units (blocks, or rows
// for the diagonal gather) are ordered by (window of 2^wl consecutive units,
// tet-code count, CZ-code count) and cut into slices of 32 / lanes units;
// `lanes` threads serve a unit.  Slice s keeps meta[s] = {first code, tet
// iterations, CZ iterations, 0}; iteration k of lane l reads
// codes[meta.x + 32 k + l] (one coalesced 128 B load per warp), the tet
// iterations first.  Lane sub of a unit takes its codes sub, sub + lanes, ...;
// missing ones are ICF_CODE_PAD.  unit[u] = {output block, row or -1}.
#define ICF_CODE_PAD 0xFFFFFFFFu
#define ICF_LAYOUT_RECORDS 0
#define ICF_LAYOUT_CONTRIB 1
#define ICF_CONTRIB_BYTES 64  // bytes per contribution record
struct icf_sell {
  int lanes = 1;
  bool natural = false;  // units in their own order (no count sort): slices of consecutive units
  int n_units = 0, n_slices = 0, slices_cap = 0;
  long long n_codes = 0, codes_cap = 0;  // code slots, padding included
  long long n_real = 0;                   // contribution codes of the units (no padding)
  int4 *meta = nullptr;
  int2 *unit = nullptr;    // merged slots of the current structure
  int2 *unit_s = nullptr;  // static slots (the lists are built once per static pattern)
  uint32_t *codes = nullptr;
};

// Row tiles of the static pattern (icf_tile.cu): the rows cut, in Morton
// order of their nodes, into tiles whose tets (those with a vertex on one of
// the tile's rows) number at most ICF_TILE_TETS.  One CTA of k_gather_tile
// stages a tile in shared memory and writes every block of its rows.
//   tiles[t]  = {first tet in ttet, tets, first slice, slices}
//   trange[t] = {first tet code, tet codes} of the tile's slices
//   ttet      = each tile's tets, ascending
//   meta[s]   = {first tet code, tet iterations, CZ iterations, first CZ code}
//   unit      = 32 per slice: {block, row or -1} (unit_s: static slots; unit:
//               merged slots of the current structure)
//   tcodes    = 16-bit tet codes (position in the tile << 4 | a << 2 | b),
//               sliced ELL: iteration k of lane l at first + 32 k + l; 0xFFFF pads
//   czcodes   = the CZ codes, sliced ELL likewise
#define ICF_TILE_TETS 384
#define ICF_TILE_CODES 8192  // tet codes of a tile, before padding
struct icf_tiles {
  bool built = false;  // for the current static pattern
  bool ok = false;     // false: some row has more tets than a tile holds
  int n_tiles = 0, n_slices = 0;
  long long n_ttet = 0, n_tcodes = 0, n_czcodes = 0, n_real = 0;
  long long n_diag_units = 0, n_off_units = 0;
  size_t smem64 = 0, smem32 = 0;  // shared memory of the largest tile
  size_t smemf64 = 0, smemf32 = 0;  // ... for the fused kernel (tets computed in place)
  int4 *tiles = nullptr;
  int2 *trange = nullptr;
  int *ttet = nullptr;
  int4 *meta = nullptr;
  int2 *unit_s = nullptr, *unit = nullptr;
  uint16_t *tcodes = nullptr;
  uint32_t *czcodes = nullptr;
};

// Workspace of the broad and narrow phases, kept across calls and grown to the
// high-water mark, so that a call allocates nothing in the usual case.
struct icf_contact_ws {
  // broad phase, per surface element (capacity b_cap)
  double *lohi = nullptr, *ext = nullptr, *tmpv = nullptr, *red = nullptr;
  int *bcnt = nullptr, *boff = nullptr;
  int4 *clo = nullptr;
  long long b_cap = 0;
  // (cell, element) entries (capacity ent_cap) and their pair counts/offsets
  unsigned long long *ek0 = nullptr, *ek1 = nullptr;
  int *ee0 = nullptr, *ee1 = nullptr, *pc = nullptr, *po = nullptr;
  long long ent_cap = 0;
  // candidate pairs before de-duplication (capacity pair_cap, padded with
  // all-ones keys that sort last)
  unsigned long long *p0 = nullptr, *p1 = nullptr;
  long long pair_cap = 0;
  // narrow phase: per pair counts/offsets and the (node, element) keys
  int *ncnt = nullptr, *noff = nullptr;
  long long ncnt_cap = 0;
  unsigned long long *nk0 = nullptr, *nk1 = nullptr;
  long long nkey_cap = 0;
  // direct contact detection: a dense grid of cells (counts, offsets,
  // cursors; capacity cell_cap) holding the surface nodes as {x, y, z, k}
  // entries (k the surface-node index; capacity gnode_cap)
  int *gcnt = nullptr, *goff = nullptr, *gcur = nullptr;
  double4 *gnode = nullptr;
  long long cell_cap = 0, gnode_cap = 0;
  // per surface node: hit counts, offsets, cursors (capacity kcap)
  int *kcnt = nullptr, *koff = nullptr, *kcur = nullptr;
  long long kcap = 0;
  // per surface element: edge-matrix inverse and first vertex (12 doubles)
  double *tinv = nullptr;
  long long tinv_cap = 0;
  // the detection grid's parameters {nx, ny, nz, C, status} and their pinned
  // host copy
  int *gp = nullptr, *h_gp = nullptr;
  // the detection's captured launches and what they were captured with
  cudaGraphExec_t det_exec = nullptr;
  std::vector<long long> det_key;
  // small device results and their pinned host copy: [0] unique count,
  // [1] impact list differs from the built one, [2] pairs before de-duplication
  int *d_small = nullptr, *h_small = nullptr;
  double *h_red = nullptr;  // pinned: the broad phase's grid reduction (7)
};

// Device MINRES solver state (icf_solve.cu).
struct icf_solver {
  long long gen = -1;  // structure generation the lower-block index belongs to
  int *lrows = nullptr, *lcols = nullptr, *lslot = nullptr;
  long long rows_cap = 0, l_cap = 0, ls_cap = 0;
  double *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr, *dinv = nullptr;
  double *w = nullptr, *w2 = nullptr;
  long long x_cap = 0, r_cap = 0, z_cap = 0, p_cap = 0, q_cap = 0, d_cap = 0, w_cap = 0, w2_cap = 0;
  double *part = nullptr, *sc = nullptr;
  double *h_sc = nullptr;  // pinned
  int n_indefinite = 0;    // diagonal blocks of the last solve preconditioned by |S|^-1
};

// Parameters the kernels read, passed by value (they live in the kernel
// parameter bank, i.e. constant memory).
struct icf_dprm {
  double lam, mu;   // Lame constants of the isotropic E
  double rho20;     // rho / 20 (consistent mass pattern)
  double dm, ds;    // Rayleigh damping (mass, stiffness)
  double nbeta, ngamma;
  double grav_rho;  // gravity * rho
  // PPR (global values; per-CZ f_tn, f_tt, deln, delt may override)
  double f_tn, f_tt, alpha, beta, rn, rt, p_m, p_n, deln, delt, pMtn, pMnt,
      gam_n, gam_t;
  double sf[9];     // sf[node*3+gp]
  double penaltyK, eps2;
};

struct icf_ctx {
  int device = 0;
  int n_sm = 148;  // multiprocessors of the device (persistent launch grids)
  cudaStream_t stream = nullptr;
  // auxiliary streams and events of the assembly's fork/join graph
  cudaStream_t aux[2] = {nullptr, nullptr};
  cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  // the assembly captured as a CUDA graph; re-captured when anything it
  // bakes in (pattern, sizes, parameters, buffers, time step) changes
  bool use_graph = true;
  cudaGraphExec_t graph_exec = nullptr;
  double graph_h = 0.0;
  unsigned long long version = 1, graph_version = 0;
  std::string err;
  icf_params prm{};
  bool have_prm = false;
  // PPR axis factors at zero opening, normal then tangential: f, d, dd and
  // the term magnitudes md, mf and rounding count k of the decision bounds
  double axis0[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  // the reference's dN, dT at zero opening (its rounding noise), normal then
  // tangential, from the host C library's pow
  double z0[2] = {0, 0};
  // the CZ kernel settles every failure comparison with the reference's
  // rounding (set while an assembly with an undecided comparison is repeated)
  bool cz_exact = false;
  double last_h = 0.0;  // time step of the last assembly
  int n_law_exact = 0;  // comparisons the last assembly settled exactly
  int precision = ICF_FP64;

  // sizes
  int n_nodes = 0, n_elem = 0, n_cz = 0, n_surf = 0, n_faces = 0;
  int N = 0;          // rows of the pattern
  int nnz_s = 0;      // static blocks
  long long n_rc = 0; // static contribution codes
  long long n_rc_off = 0; // ... of which to off-diagonal blocks
  int nnz = 0;        // merged blocks
  bool have_static = false, have_nodes = false, have_structure = false;
  bool src_identity = true;

  // topology
  int4 *d_elem = nullptr;
  int *d_cz = nullptr;
  int *d_alt = nullptr;
  int4 *d_selem = nullptr;
  int *d_adj_off = nullptr, *d_adj = nullptr, *d_faces = nullptr;
  std::vector<int> h_alt;

  // node state
  double4 *d_x0 = nullptr, *d_xc = nullptr;
  double2 *d_va = nullptr;
  double *d_u = nullptr, *d_v = nullptr, *d_a = nullptr, *d_du = nullptr;
  double *d_un = nullptr; // tentative displacement (for accept)
  double *d_h3 = nullptr; // H2D staging for n_nodes*3 fields (3 arrays)

  // CZ state
  double *d_czs = nullptr;      // current pmax[3], tmax[3]
  int *d_czfail = nullptr;      // committed failed flag
  double *d_cztent = nullptr;   // pmax_, tmax_
  int *d_czflags = nullptr;     // contact | damaged<<1 | failed<<2
  double *d_czavg = nullptr;    // avgDn, avgDt, avgTn, avgTt
  double4 *d_czprm = nullptr;   // per-CZ f_tn, f_tt, deln, delt
  bool per_cz_prm = false;

  // staging
  double4 *d_es = nullptr;
  double *d_cs = nullptr;
  double *d_ks = nullptr;
  int ks_cap = 0;

  // static pattern
  unsigned long long *d_skeys = nullptr;
  int *d_rc_off = nullptr;
  uint32_t *d_rc = nullptr;

  // gather metadata of the static pattern: start of the CZ codes per slot,
  // diagonal slot per row (-1 if none), compacted off-diagonal slots
  int *d_rc_mid = nullptr, *d_diag = nullptr, *d_offd = nullptr;
  int n_offd = 0;
  // static -> merged slot (when contact pairs add blocks) and the merged
  // positions of the contact-only blocks
  int *d_s2m = nullptr, *d_dynpos = nullptr;
  int s2m_cap = 0, dynpos_cap = 0, n_dyn = 0;
  // gather descriptors {merged position, first tet code, first CZ code, end}:
  // N per-row diagonal entries, then one per off-diagonal block (one buffer)
  int4 *d_gdesc_diag = nullptr, *d_gdesc_off = nullptr;
  int gdesc_cap = 0;
  // the gathers' sliced-ELL code lists (built from the descriptors).  With
  // split_cz the units without CZ codes (sell_off / sell_diag) and those with
  // CZ codes (sell_off_cz / sell_diag_cz) are separate lists, so the first
  // can be gathered while the CZ kernel still runs; otherwise everything is
  // in sell_off / sell_diag.
  icf_sell sell_off, sell_diag, sell_off_cz, sell_diag_cz;
  bool split_cz = false;
  // row-tile gather (one kernel for all blocks) instead of the two list gathers;
  // fused_tiles: the tile kernel computes its tets itself (no tet kernel)
  icf_tiles tiles;
  bool gather_tiles = false, fused_tiles = false;
  // the two list gathers one after the other on the main stream instead of
  // side by side
  bool serial_gathers = false;
  // touched blocks of the impacts that the off-diagonal list gather writes
  // (static, off the diagonal): their impact terms wait for that gather
  int n_crs_off = 0;
  // the gather lists exist for the current static pattern, layout and split
  // (their units in static slots; each structure only remaps the slots)
  bool lists_static = false;

  // merged pattern
  int *d_rows = nullptr, *d_cols = nullptr, *d_src = nullptr;
  int rows_cap = 0, cols_cap = 0;
  unsigned long long *d_mkeys = nullptr;

  // impacts and their contributions
  int n_imp = 0, imp_cap = 0;
  int4 *d_imp = nullptr;
  // the impact list the current merged structure was built from (-1: none);
  // a structure request with the same list keeps the structure
  int n_imp_built = -1, imp_built_cap = 0;
  int4 *d_imp_built = nullptr;
  // bumped whenever d_imp is reallocated: a kept structure (and the graph
  // captured over it) holds the d_imp pointer it was built with
  unsigned long long imp_gen = 0, imp_gen_built = 0;
  // set by the narrow phase, which compares its new list with the built one
  // on the device: imp_cmp_valid while that comparison is current
  bool imp_cmp_valid = false;
  int imp_differ = 1;
  icf_contact_ws cws;
  // per-impact classification {kind, ia, ib, 0} and {s, t, dsq, 0}; same
  // capacity as the impact staging d_ks (ks_cap)
  int n_crs = 0;                  // slots touched by impacts
  int *d_cr_slot = nullptr, *d_cr_off = nullptr;
  uint32_t *d_cr = nullptr;
  int cr_cap = 0;
  // the touched slots in k_imp_add's order: those the off-diagonal gather
  // does not write (diagonal and contact-only blocks, n_crs - n_crs_off)
  // first, then the static off-diagonal ones, so that each k_imp_add launch
  // covers its own contiguous range: per slot its records' range in d_cr,
  // the slot and, for a diagonal block, its rhs row (else -1)
  int2 *d_cr_range = nullptr;
  int *d_cr_pslot = nullptr, *d_cr_row = nullptr;
  // position in d_cr of the code (impact u, vertices a, b) at 16 u + 4 a + b,
  // or -1 (no code: an anchored vertex, or the pair taken as (b, a))
  int *d_imp_pos = nullptr;
  long long imp_pos_cap = 0;

  // narrow phase
  int n_pairs = 0, pairs_cap = 0;
  int *d_pairs = nullptr, *d_masks = nullptr;
  int *d_sgroup = nullptr;  // group (mesh) of every surface element, or null
  // surface nodes (the nodes of the surface elements, ascending) and, per
  // surface node, the surface elements holding it (ascending): the direct
  // contact detection's queries and its pair-rule check
  int *d_snode = nullptr, *d_sinc_off = nullptr, *d_sinc = nullptr;
  int n_snode = 0;
  int sgroup_bits = -1;     // bits of the largest group id; -1: none set or some negative
  bool pairs_from_broad = false;

  // node incidence lists for the node forces
  icf_node_inc tet_inc, imp_inc;

  // outputs
  double *d_vals = nullptr, *d_rhs = nullptr, *d_nodeF = nullptr;
  int vals_cap = 0;

  // counters: [0] damaged [1] failed [2] contact [3] active impacts [4] nonfinite
  // [5] undecided CZ law comparisons
  int *d_counts = nullptr;
  int *h_counts = nullptr; // pinned
  double *d_norm = nullptr;
  double *h_norm = nullptr; // pinned

  // scratch
  void *d_tmp = nullptr;
  size_t tmp_bytes = 0;

  // per-kernel timing (icf_profile_assembly): when set, the assembly runs
  // on the main stream only and each kernel is followed by an event
  struct icf_prof_state *prof = nullptr;
  // launch variants chosen by the autotuner (indices into the variant tables)
  int tune_tet = 0, tune_off = 0, tune_diag = 0, tune_cz = 0;
  // staging layout of the tet contributions:
  //   ICF_LAYOUT_RECORDS  per-tet records es[8e + ...] read at random by the
  //                       gathers through the contribution codes;
  //   ICF_LAYOUT_CONTRIB  per-contribution records written by the tet kernel
  //                       straight into the gathers' sliced-ELL positions
  //                       (d_stage_off / d_stage_diag, 64 B each, position
  //                       map d_tetpos[16 e + 4 a + b]), read as streams.
  int layout = ICF_LAYOUT_RECORDS;
  int *d_tetpos = nullptr;
  long long tetpos_cap = 0;
  void *d_stage_off = nullptr, *d_stage_diag = nullptr;
  long long stage_off_cap = 0, stage_diag_cap = 0;  // bytes
  // CZ history axes at the committed pmax/tmax (k_cz_hist), 18 doubles per CZ;
  // refilled before the next assembly whenever hist_valid is false
  double *d_czhist = nullptr;
  bool hist_valid = false;
  // linear solve; struct_gen counts structure builds
  icf_solver solver;
  long long struct_gen = 0;
};

#define ICF_PROF_MAX 16
struct icf_prof_state {
  int n = 0;
  const char *name[ICF_PROF_MAX];
  long long bytes[ICF_PROF_MAX];
  cudaEvent_t ev[ICF_PROF_MAX + 1];
};
// Records the end of the kernel just launched on `s` (no-op unless profiling).
void icf_prof_mark(icf_ctx *ctx, cudaStream_t s, const char *name, long long bytes);
// gathers (icf_gather.cu): variant tables and launchers
int icf_gather_variants(int kind);  // kind 0 off-diagonal, 1 diagonal
const char *icf_gather_variant_name(int kind, int v);
int icf_gather_variant_lanes(int v);  // lanes per row of diagonal variant v
bool icf_gather_variant_natural(int v);  // off-diagonal variant v reads natural-order lists
int icf_launch_gather_off(icf_ctx *ctx, const icf_sell &S, int variant, const double4 *es, const double *cs,
                          double sc, double mc, double lam, double mu, double *vals, cudaStream_t s);
int icf_launch_gather_diag(icf_ctx *ctx, const icf_sell &S, int variant, const double4 *es, const double *cs,
                           double sc, double mc, double lam, double mu, double *vals, double *rhs, cudaStream_t s);
// tet kernel variants (icf_assembly.cu)
int icf_tet_variants();
const char *icf_tet_variant_name(int v);
int icf_launch_tet(icf_ctx *ctx, int variant, const double4 *xc, const double2 *va, double4 *es, cudaStream_t s);
int icf_cz_variants();
const char *icf_cz_variant_name(int v);
int icf_launch_cz(icf_ctx *ctx, int variant, const double4 *xc, double *cs, cudaStream_t s);
// rebuilds the diagonal gather lists for `lanes` lanes per row (icf_pattern.cu)
int icf_build_tiles(icf_ctx *ctx);       // host-built, once per static pattern
int icf_remap_tiles(icf_ctx *ctx);       // unit slots for the current structure
void icf_free_tiles(icf_ctx *ctx);
int icf_gather_tile_setup(icf_ctx *ctx);
bool icf_tiles_active(const icf_ctx *ctx);
int icf_launch_gather_tile(icf_ctx *ctx, const double4 *es, const double *cs, double sc, double mc, double lam,
                           double mu, double *vals, double *rhs, cudaStream_t s);
// the fused row-tile kernel (tets computed in shared memory) over node state xc, va
int icf_launch_tile_fused(icf_ctx *ctx, const double4 *xc, const double2 *va, const double *cs, double sc,
                          double mc, double *vals, double *rhs, cudaStream_t s);
inline bool icf_fused_active(const icf_ctx *ctx) { return ctx->fused_tiles && icf_tiles_active(ctx); }
int icf_rebuild_lists(icf_ctx *ctx);  // both gathers' lists for the current layout and split
int icf_remap_lists(icf_ctx *ctx);    // their units' slots for the current structure
// 1 for a merged slot that the off-diagonal gather writes: static, off the diagonal
__host__ __device__ inline bool icf_off_static(const unsigned long long *mkey, const int *src, int identity, int s) {
  const unsigned long long k = mkey[s];
  return (identity || src[s] >= 0) && (k >> 32) != (k & 0xffffffffull);
}  // both gathers' lists for the current layout and split
int icf_rebuild_sell_diag(icf_ctx *ctx, int lanes);
int icf_rebuild_sell_off(icf_ctx *ctx, bool natural);
// position map and zeroed contribution staging for the current lists
int icf_build_contrib(icf_ctx *ctx);
int icf_ensure_cz_hist(icf_ctx *ctx, cudaStream_t s);
// the cohesive law alone on device arrays (icf_cz_law_eval): in[4n], prm[n]
// or null, out[7n], fl[2n]
int icf_launch_law_eval(icf_ctx *ctx, int n, const double *in, const double4 *prm, double *out, int *fl);
// after an assembly left a law comparison undecided (counts[5]), repeats it
// with the exact CZ kernel; `rerun` enqueues the same assembly again
int icf_settle_law(icf_ctx *ctx, const std::function<int()> &rerun);
int icf_solve_impl(icf_ctx *ctx, double rel_tol, int max_iter, int *iters, double *relres);
void icf_free_solver(icf_ctx *ctx);
int icf_launch_sumsq(icf_ctx *ctx, const double *d_x, long long n);
int icf_broad_phase_impl(icf_ctx *ctx, double pad, const int *d_group, int *n_pairs_out);
void icf_free_contact_ws(icf_ctx *ctx);
int icf_autotune_impl(icf_ctx *ctx, double h, int reps, icf_tune_report *out);
int icf_set_variant_impl(icf_ctx *ctx, int kind, int variant);
int icf_profile_assembly_impl(icf_ctx *ctx, double h, int reps, int *n, const char **names,
                              long long *bytes, double *ms);

// ---- error plumbing ---------------------------------------------------------
int icf_fail(icf_ctx *ctx, int code, const std::string &msg);
#define ICF_CUDA(ctx, call)                                                    \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess)                                                     \
      return icf_fail((ctx), ICF_ERR_CUDA,                                     \
                      std::string(#call) + ": " + cudaGetErrorString(e_));     \
  } while (0)

int icf_scratch(icf_ctx *ctx, size_t bytes);
#define ICF_TRY_RC(call)        \
  do {                          \
    const int rc_ = (call);     \
    if (rc_ != ICF_OK) return rc_; \
  } while (0)

inline unsigned icf_blocks(long long n, int bs) {
  return (unsigned)((n + bs - 1) / bs);
}

icf_dprm icf_make_dprm(const icf_ctx *ctx);

// ---- kernels and launchers implemented in the .cu files ---------------------
int icf_build_static_pattern(icf_ctx *ctx);
int icf_build_merged_pattern(icf_ctx *ctx);
int icf_launch_assembly(icf_ctx *ctx, double h);
int icf_launch_node_force(icf_ctx *ctx);
int icf_run_narrow_phase(icf_ctx *ctx, int n_pairs, int *n_impacts);
int icf_launch_count_damaged(icf_ctx *ctx, int *d_count);
int icf_finish_impacts(icf_ctx *ctx, const unsigned long long *keys, int total, const int *d_n, int eb,
                       int *n_impacts);
// broad phase, narrow phase and closest face in one, without the pair list
// (icf_broad.cu): the impact list icf_run_narrow_phase gives on the pairs of
// icf_broad_phase_impl with the same pad and groups
int icf_detect_contacts_impl(icf_ctx *ctx, double pad, const int *d_group, int *n_impacts);
int icf_launch_pcsr(icf_ctx *ctx, int kind, int *d_out);
int icf_launch_pack_nodes(icf_ctx *ctx, const double *d_un, const double *d_vn,
                          const double *d_an);
int icf_launch_infer(icf_ctx *ctx, double h);
int icf_launch_add_dx(icf_ctx *ctx, const double *d_dx);
int icf_launch_accept(icf_ctx *ctx, double h);
int icf_launch_commit_cz(icf_ctx *ctx);
int icf_launch_imp_unit(icf_ctx *ctx, cudaStream_t stream);
int icf_launch_imp_deriv(icf_ctx *ctx, cudaStream_t stream);
int icf_get_node_inc(icf_ctx *ctx, icf_node_inc *tets, icf_node_inc *imps);

// Buffers of one assembly when the caller, not the context, provides them
// (the allocation-free entry point, icf_noalloc.cu).
struct icf_asm_bufs {
  const double *un, *vn, *an;  // node state in, n_nodes*3 each
  double4 *xc;                 // n_nodes
  double2 *va;                 // 3*n_nodes
  double4 *es;                 // 8*n_elem
  double *cs;                  // ICF_CZ_STAGE*n_cz
  double *ks;                  // ICF_IMP_STAGE*n_imp
  double *vals, *rhs;          // outputs, nnz*9 and N*3
};
int icf_enqueue_assembly_bufs(icf_ctx *ctx, double h, const icf_asm_bufs &B, cudaStream_t s);
int icf_launch_imp_unit_bufs(icf_ctx *ctx, const double4 *xc, double *ks, cudaStream_t stream);
int icf_launch_imp_deriv_bufs(icf_ctx *ctx, const double4 *xc, double *ks, cudaStream_t stream);
