// icf_noalloc.cu -- an assembly entry point that allocates no device memory.
//
// Some callers cannot call cudaMalloc while they assemble: a host that hands
// out every byte of device memory from its own pre-sized pool, or a solver
// loop that must not touch the allocator (and its implicit synchronisation)
// between iterations.  icf_assemble_noalloc serves them.  It takes the node
// state and the output arrays as device pointers from the caller and keeps
// every temporary of the assembly -- the packed node state and the tet, CZ and
// impact staging -- in one fixed array declared below, which each GPU that
// loads the library holds until the process exits.  It calls no cudaMalloc,
// cudaFree or allocating library routine.
//
// The array's size is fixed at ICF_NOALLOC_BYTES (8 MiB).  A model whose
// temporaries do not fit (80 B per node, 256 B per tet, 384 B per CZ, 1056 B
// per impact, each section rounded up to 256 B) is rejected with
// ICF_ERR_SIZE and a message giving both numbers.
//
// All calls on a device share the one array and it keeps the contents of the
// last call; everything a call reads from it is written earlier in the same
// call, and the counters that must start at zero live in the context and are
// cleared on the stream first.  Calls whose work overlaps on the GPU (two
// threads, two contexts on one device, or two streams) race on the array; the
// entry point is synchronous, so calls made one after another from one thread
// do not overlap.
//
// The host never dereferences `g_noalloc_scratch`: in host code that name
// stands for the device variable and is not its address.  The device address
// is looked up once per device with cudaGetSymbolAddress, with that device
// current, the first time the entry point runs on it; make that first call
// before any stream capture.
#include <mutex>

#include "icf_internal.cuh"

#define ICF_NOALLOC_BYTES (8u << 20)
#define ICF_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) unsigned char g_noalloc_scratch[ICF_NOALLOC_BYTES];

namespace {
std::mutex g_noalloc_mu;
void *g_noalloc_ptr[ICF_NOALLOC_MAX_DEVICES] = {};

size_t round256(size_t b) { return (b + 255) & ~size_t(255); }
}  // namespace

extern "C" int icf_assemble_noalloc(icf_ctx *ctx, double h, const double *d_un, const double *d_vn,
                                    const double *d_an, double *d_vals, double *d_rhs,
                                    icf_counts *counts) {
  if (!ctx) return ICF_ERR_ARG;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return icf_fail(ctx, ICF_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  if (!ctx->have_prm) return icf_fail(ctx, ICF_ERR_STATE, "icf_set_constants first");
  if (!ctx->have_structure) return icf_fail(ctx, ICF_ERR_STATE, "icf_create_structure first");
  if (!(h > 0)) return icf_fail(ctx, ICF_ERR_ARG, "time step must be positive");
  if (!d_un || !d_vn || !d_an || !d_vals || !d_rhs)
    return icf_fail(ctx, ICF_ERR_ARG, "null device buffer");
  if (ctx->device < 0 || ctx->device >= ICF_NOALLOC_MAX_DEVICES)
    return icf_fail(ctx, ICF_ERR_ARG, "device index beyond the scratch table");

  // sections of the scratch array for this model
  const size_t n = (size_t)ctx->n_nodes;
  const size_t b_xc = round256(sizeof(double4) * n), b_va = round256(sizeof(double2) * 3 * n);
  const size_t b_es = round256(sizeof(double4) * 8 * (size_t)ctx->n_elem);
  const size_t b_cs = round256(sizeof(double) * ICF_CZ_STAGE * (size_t)ctx->n_cz);
  const size_t b_ks = round256(sizeof(double) * ICF_IMP_STAGE * (size_t)ctx->n_imp);
  const size_t need = b_xc + b_va + b_es + b_cs + b_ks;
  if (need > ICF_NOALLOC_BYTES)
    return icf_fail(ctx, ICF_ERR_SIZE,
                    "model needs " + std::to_string(need) + " bytes of scratch; the allocation-free "
                    "entry point has " + std::to_string((size_t)ICF_NOALLOC_BYTES));

  // device address of the array, looked up once per device
  void *base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[ctx->device]) {
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p)
        return icf_fail(ctx, ICF_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_noalloc_ptr[ctx->device] = p;
    }
    base = g_noalloc_ptr[ctx->device];
  }

  unsigned char *p = static_cast<unsigned char *>(base);
  icf_asm_bufs B;
  B.un = d_un;
  B.vn = d_vn;
  B.an = d_an;
  B.xc = reinterpret_cast<double4 *>(p);
  p += b_xc;
  B.va = reinterpret_cast<double2 *>(p);
  p += b_va;
  B.es = reinterpret_cast<double4 *>(p);
  p += b_es;
  B.cs = reinterpret_cast<double *>(p);
  p += b_cs;
  B.ks = reinterpret_cast<double *>(p);
  B.vals = d_vals;
  B.rhs = d_rhs;

  const int rc = icf_enqueue_assembly_bufs(ctx, h, B, ctx->stream);
  if (rc != ICF_OK) return rc;
  e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return icf_fail(ctx, ICF_ERR_CUDA, std::string("assembly: ") + cudaGetErrorString(e));
  ctx->n_law_exact = 0;
  const int rs = icf_settle_law(ctx, [&] { return icf_enqueue_assembly_bufs(ctx, h, B, ctx->stream); });
  if (rs != ICF_OK) return rs;
  if (counts) {
    counts->nElems = ctx->n_elem;
    counts->nCZ = ctx->n_cz;
    counts->nCZDamaged = ctx->h_counts[0];
    counts->nCZFailedThisStep = ctx->h_counts[1];
    counts->nCZContact = ctx->h_counts[2];
    counts->nImpacts = ctx->n_imp;
    counts->nImpactsActive = ctx->h_counts[3];
    counts->nonFinite = ctx->h_counts[4];
    counts->nLawExact = ctx->n_law_exact;
  }
  if (ctx->h_counts[4]) return icf_fail(ctx, ICF_ERR_NUMERIC, "non-finite value in the assembled rhs");
  return ICF_OK;
}
