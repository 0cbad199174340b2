// icf_tune.cu -- the launch-variant autotuner.
//
// The tet kernel and the two gathers each come in several launch variants
// (registers per thread, codes per iteration, loads through registers or
// cp.async, lanes per row).  Every variant computes the same values.  Which one
// is fastest depends on the model's size and on its code-count
// distribution, so the tuner times each variant on the model at hand (device
// events around `reps` back-to-back launches on the context stream, after one
// untimed launch) and keeps the fastest.  The choice stays with the context
// and is baked into the assembly graph at its next capture.
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
                          : (kind == 1 ? icf_gather_variants(0) : (kind == 2 ? icf_gather_variants(1) : 2));
  if (kind < 0 || kind > 3 || variant < 0 || variant >= n)
    return icf_fail(ctx, ICF_ERR_ARG, "icf_set_variant: kind 0..3 and a variant index of that kind");
  if (kind == 3) ctx->layout = variant;
  if (kind == 0) ctx->tune_tet = variant;
  if (kind == 1) ctx->tune_off = variant;
  if (kind == 2) {
    ctx->tune_diag = variant;
    const int lanes = icf_gather_variant_lanes(variant);
    if (ctx->have_structure && lanes != ctx->sell_diag.lanes) ICF_TRY_RC(icf_rebuild_sell_diag(ctx, lanes));
  }
  ctx->version++;
  return ICF_OK;
}

int icf_autotune_impl(icf_ctx *ctx, double h, int reps, icf_tune_report *out) {
  if (out) memset(out, 0, sizeof(*out));
  // one assembly so that every staging buffer holds this model's values
  ICF_TRY_RC(icf_launch_assembly(ctx, h));
  ICF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  timer t;
  ICF_CUDA(ctx, cudaEventCreate(&t.a));
  ICF_CUDA(ctx, cudaEventCreate(&t.b));
  const icf_dprm P = icf_make_dprm(ctx);
  const double nb = ctx->prm.NewmarkBeta, ng = ctx->prm.NewmarkGamma;
  const double sc = 1.0 + ctx->prm.dampingStiffness * ng / (h * nb);
  const double mc = (1.0 / (h * h) + ctx->prm.dampingMass * ng / h) / nb * (ctx->prm.rho / 20.0);

  // staging layout: whole assemblies (graph launches) with each layout
  {
    const char *names[2] = {"per-tet records", "per-contribution stream"};
    double best = 1e30;
    int bl = ctx->layout;
    for (int l = 0; l < 2; l++) {
      ctx->layout = l;
      ctx->version++;
      double ms = 0;
      ICF_TRY_RC(time_launches(ctx, t, reps, [&] { return icf_launch_assembly(ctx, h); }, &ms));
      report(out, "layout", names[l], ms);
      if (ms < best) best = ms, bl = l;
    }
    ctx->layout = bl;
    ctx->version++;
    mark_chosen(out, "layout", names[bl]);
    ICF_TRY_RC(icf_launch_assembly(ctx, h));
    ICF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  // tets
  if (ctx->n_elem > 0) {
    double best = 1e30;
    int bv = 0;
    for (int v = 0; v < icf_tet_variants(); v++) {
      double ms = 0;
      ICF_TRY_RC(time_launches(ctx, t, reps, [&] { return icf_launch_tet(ctx, v, ctx->d_xc, ctx->d_va, ctx->d_es, ctx->stream); }, &ms));
      report(out, "k_tet_unit", icf_tet_variant_name(v), ms);
      if (ms < best) best = ms, bv = v;
    }
    ctx->tune_tet = bv;
    mark_chosen(out, "k_tet_unit", icf_tet_variant_name(bv));
  }
  // off-diagonal gather
  if (ctx->sell_off.n_slices > 0) {
    double best = 1e30;
    int bv = 0;
    for (int v = 0; v < icf_gather_variants(0); v++) {
      double ms = 0;
      ICF_TRY_RC(time_launches(ctx, t, reps, [&] {
        return icf_launch_gather_off(ctx, v, ctx->d_es, ctx->d_cs, sc, mc, P.lam, P.mu, ctx->d_vals, ctx->stream);
      }, &ms));
      report(out, "k_gather_off", icf_gather_variant_name(0, v), ms);
      if (ms < best) best = ms, bv = v;
    }
    ctx->tune_off = bv;
    mark_chosen(out, "k_gather_off", icf_gather_variant_name(0, bv));
  }
  // diagonal gather: each lanes-per-row layout needs its own lists
  if (ctx->N > 0) {
    double best = 1e30;
    int bv = 0;
    const int lanes_list[3] = {2, 4, 8};
    for (int li = 0; li < 3; li++) {
      bool any = false;
      for (int v = 0; v < icf_gather_variants(1); v++) any |= icf_gather_variant_lanes(v) == lanes_list[li];
      if (!any) continue;
      ICF_TRY_RC(icf_rebuild_sell_diag(ctx, lanes_list[li]));
      // new list positions: the contribution staging is refilled by the tets
      ICF_TRY_RC(icf_launch_tet(ctx, ctx->tune_tet, ctx->d_xc, ctx->d_va, ctx->d_es, ctx->stream));
      for (int v = 0; v < icf_gather_variants(1); v++) {
        if (icf_gather_variant_lanes(v) != lanes_list[li]) continue;
        double ms = 0;
        ICF_TRY_RC(time_launches(ctx, t, reps, [&] {
          return icf_launch_gather_diag(ctx, v, ctx->d_es, ctx->d_cs, sc, mc, P.lam, P.mu, ctx->d_vals,
                                        ctx->d_rhs, ctx->stream);
        }, &ms));
        report(out, "k_gather_diag", icf_gather_variant_name(1, v), ms);
        if (ms < best) best = ms, bv = v;
      }
    }
    ctx->tune_diag = bv;
    if (ctx->sell_diag.lanes != icf_gather_variant_lanes(bv))
      ICF_TRY_RC(icf_rebuild_sell_diag(ctx, icf_gather_variant_lanes(bv)));
    mark_chosen(out, "k_gather_diag", icf_gather_variant_name(1, bv));
  }
  ctx->version++;
  // leave the outputs of a complete assembly behind
  ICF_TRY_RC(icf_launch_assembly(ctx, h));
  return icf_read_counts(ctx, nullptr);
}
