// icf_tune.cu -- the launch-variant autotuner.
//
// The tet kernel, the CZ kernel and the two gathers each come in several
// launch variants (registers per thread, codes per iteration, lanes per row),
// and the tet contributions have two staging layouts.  Every variant computes
// the same values.  Which one is fastest depends on the model's size, on its
// code-count distribution and on what runs beside it in the graph, so the
// tuner times whole assemblies on the model at hand (device events around
// `reps` back-to-back graph launches on the context stream, after one untimed
// launch that re-captures the graph) and keeps the fastest choice of each
// kind in turn.  The choice stays with the context.
#include <cstring>
#include <string>

#include "icf_internal.cuh"

namespace {

struct timer {
  cudaEvent_t a = nullptr, b = nullptr;
  ~timer() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

void report(icf_tune_report *out, const char *kernel, const char *variant, double ms) {
  if (!out || out->n >= ICF_MAX_TUNE) return;
  const int i = out->n++;
  strncpy(out->kernel[i], kernel, sizeof(out->kernel[i]) - 1);
  strncpy(out->variant[i], variant, sizeof(out->variant[i]) - 1);
  out->ms[i] = ms;
  out->chosen[i] = 0;
}

void mark_chosen(icf_tune_report *out, const char *kernel, const char *variant) {
  if (!out) return;
  for (int i = 0; i < out->n; i++)
    if (!strcmp(out->kernel[i], kernel) && !strcmp(out->variant[i], variant)) out->chosen[i] = 1;
}

}  // namespace

// Mean device time of `reps` launches of `launch` (one more, untimed, first).
template <typename F>
static int time_launches(icf_ctx *ctx, timer &t, int reps, F launch, double *ms) {
  ICF_TRY_RC(launch());
  ICF_CUDA(ctx, cudaEventRecord(t.a, ctx->stream));
  for (int r = 0; r < reps; r++) ICF_TRY_RC(launch());
  ICF_CUDA(ctx, cudaEventRecord(t.b, ctx->stream));
  ICF_CUDA(ctx, cudaEventSynchronize(t.b));
  float f = 0.f;
  ICF_CUDA(ctx, cudaEventElapsedTime(&f, t.a, t.b));
  *ms = f / reps;
  return ICF_OK;
}

int icf_set_variant_impl(icf_ctx *ctx, int kind, int variant) {
  const int n = kind == 0 ? icf_tet_variants()
                          : kind == 1 ? icf_gather_variants(0)
                          : kind == 2 ? icf_gather_variants(1)
                          : kind == 3 ? 2
                          : kind == 5 ? 2
                          : kind == 6 ? 3
                          : kind == 7 ? 2
                                      : icf_cz_variants();
  if (kind < 0 || kind > 7 || variant < 0 || variant >= n)
    return icf_fail(ctx, ICF_ERR_ARG, "icf_set_variant: kind 0..7 and a variant index of that kind");
  if (kind == 7) ctx->serial_gathers = variant == 1;
  if (kind == 6) {
    ctx->gather_tiles = variant >= 1;
    if (ctx->fused_tiles != (variant == 2)) ctx->version++;
    ctx->fused_tiles = variant == 2;
    if (ctx->gather_tiles && ctx->have_structure && !ctx->tiles.built) {
      ICF_TRY_RC(icf_build_tiles(ctx));
      ICF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
  }
  if (kind == 3 || kind == 5) {
    // the staging layout and the split decide which lists exist
    const bool changed = kind == 3 ? ctx->layout != variant : ctx->split_cz != (variant == 1);
    if (kind == 3) ctx->layout = variant;
    else ctx->split_cz = variant == 1;
    if (changed && ctx->have_structure) {
      ICF_TRY_RC(icf_rebuild_lists(ctx));
      ICF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
  }
  if (kind == 4) ctx->tune_cz = variant;
  if (kind == 0) ctx->tune_tet = variant;
  if (kind == 1) {
    ctx->tune_off = variant;
    const bool nat = icf_gather_variant_natural(variant);
    if (ctx->have_structure && nat != ctx->sell_off.natural) ICF_TRY_RC(icf_rebuild_sell_off(ctx, nat));
  }
  if (kind == 2) {
    ctx->tune_diag = variant;
    const int lanes = icf_gather_variant_lanes(variant);
    if (ctx->have_structure && lanes != ctx->sell_diag.lanes) ICF_TRY_RC(icf_rebuild_sell_diag(ctx, lanes));
  }
  ctx->version++;
  return ICF_OK;
}

// Coordinate descent over the launch choices, each candidate judged by the
// time of whole assemblies (the captured graph, re-captured per candidate).
// Timing kernels alone misleads: the graph runs the tet, CZ and impact
// kernels concurrently, and a variant that wins alone (say, a CZ kernel that
// packs more blocks per SM) can slow its neighbours down more than it gains.
int icf_autotune_impl(icf_ctx *ctx, double h, int reps, icf_tune_report *out) {
  if (out) memset(out, 0, sizeof(*out));
  timer t;
  ICF_CUDA(ctx, cudaEventCreate(&t.a));
  ICF_CUDA(ctx, cudaEventCreate(&t.b));
  auto assembly_ms = [&](double *ms) {
    ctx->version++;  // re-capture with the candidate's kernels
    return time_launches(ctx, t, reps, [&] { return icf_launch_assembly(ctx, h); }, ms);
  };
  int split = ctx->split_cz ? 1 : 0, tiles = ctx->fused_tiles ? 2 : (ctx->gather_tiles ? 1 : 0),
      serial = ctx->serial_gathers ? 1 : 0;
  struct kind_desc {
    const char *name;
    int kind, n;
    int *cur;
  };
  const kind_desc kinds[] = {
      {"layout", 3, 2, &ctx->layout},
      {"gather", 6, 3, &tiles},
      {"split", 5, ctx->n_cz > 0 ? 2 : 0, &split},
      {"streams", 7, 2, &serial},
      {"k_tet_unit", 0, ctx->n_elem > 0 ? icf_tet_variants() : 0, &ctx->tune_tet},
      {"k_cz_gp", 4, ctx->n_cz > 0 ? icf_cz_variants() : 0, &ctx->tune_cz},
      {"k_gather_off", 1, ctx->n_offd > 0 ? icf_gather_variants(0) : 0, &ctx->tune_off},
      {"k_gather_diag", 2, ctx->N > 0 ? icf_gather_variants(1) : 0, &ctx->tune_diag},
  };
  const char *layout_names[2] = {"per-tet records", "per-contribution stream"};
  const char *split_names[2] = {"one list per gather", "CZ-free units apart"};
  const char *gather_names[3] = {"off-diagonal + diagonal lists", "row tiles", "fused row tiles"};
  const char *stream_names[2] = {"gathers side by side", "gathers one after other"};
  for (const kind_desc &k : kinds) {
    if (k.n < 2) continue;
    // the list gathers' choices do not matter while the tiled gather runs
    if ((k.kind == 1 || k.kind == 2 || k.kind == 5 || k.kind == 7) && icf_tiles_active(ctx)) continue;
    // the fused tiles compute the tets themselves: no tet kernel to tune
    if (k.kind == 0 && icf_fused_active(ctx)) continue;
    // the stream placement matters only for one list per gather
    if (k.kind == 7 && ctx->split_cz && ctx->layout == ICF_LAYOUT_RECORDS) continue;
    // nor the tiled gather under the per-contribution layout
    if (k.kind == 6 && ctx->layout != ICF_LAYOUT_RECORDS) continue;
    double best = 1e30;
    int bv = *k.cur;
    for (int v = 0; v < k.n; v++) {
      ICF_TRY_RC(icf_set_variant_impl(ctx, k.kind, v));
      double ms = 0;
      ICF_TRY_RC(assembly_ms(&ms));
      const char *vn = k.kind == 3 ? layout_names[v]
                       : k.kind == 5 ? split_names[v]
                       : k.kind == 6 ? gather_names[v]
                       : k.kind == 7 ? stream_names[v]
                       : k.kind == 0 ? icf_tet_variant_name(v)
                       : k.kind == 4 ? icf_cz_variant_name(v)
                                     : icf_gather_variant_name(k.kind == 1 ? 0 : 1, v);
      report(out, k.name, vn, ms);
      if (ms < best) best = ms, bv = v;
    }
    ICF_TRY_RC(icf_set_variant_impl(ctx, k.kind, bv));
    const char *vn = k.kind == 3 ? layout_names[bv]
                     : k.kind == 5 ? split_names[bv]
                     : k.kind == 6 ? gather_names[bv]
                     : k.kind == 7 ? stream_names[bv]
                     : k.kind == 0 ? icf_tet_variant_name(bv)
                     : k.kind == 4 ? icf_cz_variant_name(bv)
                                   : icf_gather_variant_name(k.kind == 1 ? 0 : 1, bv);
    mark_chosen(out, k.name, vn);
  }
  ctx->version++;
  // leave the outputs of a complete assembly behind
  ICF_TRY_RC(icf_launch_assembly(ctx, h));
  return icf_read_counts(ctx, nullptr);
}
