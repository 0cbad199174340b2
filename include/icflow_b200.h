/* icflow_b200.h -- C ABI of the B200 (sm_100a) assembly path for icFlow.
 *
 * This library replaces the ManagedCUDA/PTX layer of icFlow, i.e. the C#
 * class GPU_Functionality (v3Library/Simulation/GPU/GPU_Functionality.cs:13)
 * together with the sparsity-pattern builder CSRDictionary
 * (v3Library/Simulation/LinearSystem/CSRDictionary.cs:17) and the Newmark
 * node kinematics of Node (v3Library/Geometry/Node.cs:62-97).  It follows the
 * in-repo precedent of a Cdecl C-ABI DLL called through P/Invoke
 * (LinearSystem.cs:45-46 -> PardisoLoader2/dllmain.cpp:30).
 *
 * Conventions
 *  - Every function returns int: ICF_OK (0) or a negative ICF_ERR_* code;
 *    icf_last_error() gives a message.  Nothing aborts, nothing throws.
 *  - Host buffers belong to the caller and are used only during the call.
 *  - Node fields are arrays of n_nodes x 3 doubles (x, y, z per node), in
 *    MeshCollection.allNodes order (globalNodeId).  Unit node lists are
 *    n x 4 (tets, impacts) or n x 6 (cohesive zones) ints of global node ids.
 *  - alt_id[node] is the row of the node in the linear system (Node.altId),
 *    -1 for anchored nodes (ImplicitModel3.cs:62-73).
 *  - Calls on one context must come from one thread at a time; distinct
 *    contexts are independent.  Each call makes its device current.
 *  - Results are deterministic: no floating-point atomics are used, so two
 *    runs on the same input give bit-identical matrices.
 */
#ifndef ICFLOW_B200_H
#define ICFLOW_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define ICF_OK 0
#define ICF_ERR_ARG (-1)      /* null pointer, bad index, bad count */
#define ICF_ERR_SIZE (-2)     /* buffer or capacity too small, unit limit */
#define ICF_ERR_CUDA (-3)     /* CUDA runtime error */
#define ICF_ERR_STATE (-4)    /* call order (e.g. assemble before structure) */
#define ICF_ERR_NUMERIC (-5)  /* NaN/Inf produced on the device */
#define ICF_ERR_NODEVICE (-6) /* no usable sm_100 device */

typedef struct icf_ctx icf_ctx;

/* Mirror of ModelPrms (v3Library/Simulation/DataSheets/ModelPrms.cs);
 * field names kept.  The block after "derived" is filled by
 * icf_params_derive (ModelPrms.SetComputedVariables, :237-322). */
typedef struct icf_params {
  double InitialTimeStep;
  /* material, :133-156 */
  double Y, nu, rho, dampingMass, dampingStiffness, gravity;
  /* integration, :177-209 */
  double NewmarkBeta, NewmarkGamma;
  double ConvergenceEpsilon, ConvergenceCutoff;
  double maxDamagePerStep, maxFailPerStep;
  int maxIterations, minIterations;
  /* cohesive zones, :37-65 */
  double alpha, beta, lambda_n, lambda_t, phi_n, phi_t, sigma_max, tau_max;
  /* collisions, :158-175 (CollisionScheme: 0 None, 1 Everything) */
  int CollisionScheme;
  double penaltyK, DistanceEpsilon;
  /* derived */
  double E[36];  /* E[i*6+j], isotropic elasticity, engineering shear */
  double M[144]; /* M[i*12+j], consistent mass pattern (times volume) */
  double sf[9];  /* sf[node*3+gp] */
  double B[162]; /* B[(gp*3+coord)*18+dof] */
  double G_fn, G_ft, f_tn, f_tt, rn, rt, p_m, p_n, deln, delt, pMtn, pMnt,
      gam_n, gam_t;
  double nThreshold, tThreshold;
} icf_params;

/* Arithmetic of the element and CZ Hessians.  FP64 everywhere (ICF_FP64) or
 * FP32 Hessians with FP64 rotation, near-separation cohesive law and FP64
 * accumulation (ICF_FP32_MIXED). */
#define ICF_FP64 0
#define ICF_FP32_MIXED 1

/* Per-assembly counters (FrameInfo fields set by AssembleElemsAndCZs,
 * GPU_Functionality.cs:444-475, and NarrowPhaseCollisionDetection). */
typedef struct icf_counts {
  int nElems;            /* elastic elements assembled */
  int nCZ;               /* non-failed CZs assembled */
  int nCZDamaged;        /* Sum(TENTATIVE_DAMAGED) */
  int nCZFailedThisStep; /* Sum(TENTATIVE_FAILED) */
  int nCZContact;        /* CZs with a Gauss point in contact */
  int nImpacts;          /* impacts in the current structure */
  int nImpactsActive;    /* impacts that produced a penalty response */
  int nonFinite;         /* 1 if a NaN/Inf reached the matrix or rhs */
  int nLawExact;         /* CZ Gauss points whose failure test lay within
                            rounding of its threshold; the assembly was then
                            repeated with the reference's rounding for them
                            (0 in practice; no reference counterpart) */
} icf_counts;

/* Device buffers, for callers that chain device work (graphs, solvers).
 * Pointers stay valid until the next call that changes the pattern size. */
typedef struct icf_device_buffers {
  double *vals;    /* nnz*9: block s at vals[9s], row-major 3x3 */
  double *rhs;     /* N*3 */
  int *csr_rows;   /* N+1 */
  int *csr_cols;   /* nnz */
  void *stream;    /* cudaStream_t used by the context */
  int N, nnz;
} icf_device_buffers;

/* ---- context, GPU_Functionality(int deviceID) :112-137 ----------------- */
int icf_create(int device, icf_ctx **out);
int icf_destroy(icf_ctx *ctx);
const char *icf_last_error(const icf_ctx *ctx);
/* Library version string, e.g. "icflow_b200 1.0 sm_100a". */
const char *icf_version(void);

/* ---- parameters, ModelPrms.SetComputedVariables :237-322 ---------------- */
/* Host only; fills the derived block of *p. */
int icf_params_derive(icf_params *p);
/* SetConstants, GPU_Functionality.cs:151-194 (derives, then uploads). */
int icf_set_constants(icf_ctx *ctx, const icf_params *p);
int icf_set_precision(icf_ctx *ctx, int precision);
/* Per-CZ strengths (extension of cz_constants.h:7, which is global in the
 * reference): sigma_max[c], tau_max[c] for every CZ; NULL restores the
 * global values.  deln/delt are derived per CZ. */
int icf_set_cz_strength(icf_ctx *ctx, int n_czs, const double *sigma_max,
                        const double *tau_max);

/* ---- static data, TransferStaticDataToDevice :255-302 ------------------- */
/* Mesh topology and the tables the narrow phase needs:
 *   elems[n_elems*4]        elastic elements (MeshCollection.elasticElements)
 *   czs[n_czs*6]            all CZs (vrts[0..5], CZ.cs:488)
 *   alt_id[n_nodes]         row per node, -1 anchored
 *   x0[n_nodes*3]           rest coordinates
 *   surface_elems[n_surface*4]                 (MeshCollection.surfaceElements)
 *   adj_offsets[n_surface+1], adj_faces[...]   Element.adjFaces in order
 *   faces[n_faces*3]        MeshCollection.allFaces vertices
 * The static sparsity pattern (elements + CZs, MeshCollection.cs:91-109) is
 * built here on the device.  n_surface may be 0 (no contact). */
int icf_transfer_static(icf_ctx *ctx, int n_nodes, const double *x0,
                        const int *alt_id, int n_elems, const int *elems,
                        int n_czs, const int *czs, int n_surface,
                        const int *surface_elems, const int *adj_offsets,
                        const int *adj_faces, int n_faces, const int *faces);

/* ---- per-iteration node state, TransferNodesToGPU :307-343 -------------- */
/* un, vn, an: tentative displacement, velocity, acceleration (Node.un*, vn*,
 * an*).  The current position x0 + un is formed on the device. */
int icf_transfer_nodes(icf_ctx *ctx, int n_nodes, const double *un,
                       const double *vn, const double *an);

/* ---- CZ damage state, TransferPCSR :374-413 ----------------------------- */
/* Current pmax[n*3], tmax[n*3] and failed[n] of every CZ.  Failed CZs are
 * skipped by the assembly (the reference drops them from nonFailedCZs). */
int icf_transfer_cz_state(icf_ctx *ctx, int n_czs, const double *pmax,
                          const double *tmax, const int *failed);

/* ---- contact, NarrowPhaseCollisionDetection :539-616 -------------------- */
/* pairs[n_pairs*2]: surface-element ids from the broad phase.  Runs the
 * vertex-inclusion test, expands the masks into the set of (node, element)
 * tuples (ascending by node, then element) and resolves each tuple to its
 * closest adjacent face.  The impacts become part of the next structure. */
int icf_narrow_phase(icf_ctx *ctx, int n_pairs, const int *pairs,
                     int *n_impacts);
/* Broad phase on the device (replaces the host k-DOP BVH, BVHT.cs:29-77,
 * BVHN.cs:39-194, whose element-pair list NarrowPhaseCollisionDetection
 * receives): surface-element pairs a < b whose axis-aligned boxes at the
 * current positions, widened by pad, overlap, that share no node and where a
 * vertex of one lies in the other's box; with groups (e.g. the mesh of each
 * surface element, icf_set_surface_groups) only pairs of different groups.
 * Like the reference's tree, which holds every surface element of every
 * mesh, pairs of one mesh qualify by default.  The pairs stay on the device:
 * icf_narrow_phase(ctx, -1, NULL, &n) uses them; icf_get_pairs copies them
 * out (pairs[n*2], ascending). */
int icf_set_surface_groups(icf_ctx *ctx, int n_surface, const int *group);
int icf_broad_phase(icf_ctx *ctx, double pad, int *n_pairs);
/* Non-failed CZs of the committed state damaged at the level _acceptFrame
 * counts (ImplicitModel3.cs:304-317 with CZ.damagedAtLevel, CZ.cs:13-16):
 * pmax of the first Gauss point above deln * lambda_n or tmax above
 * delt * lambda_t (per-CZ deln, delt with per-CZ strengths).  The accepted
 * frame's nCZDamaged, against which _checkDamage measures a step's new
 * damage. */
int icf_count_damaged(icf_ctx *ctx, int *n_damaged);
/* Broad phase, narrow phase and closest face in one call, without the pair
 * list (no reference counterpart; it stands for BVH self-collision +
 * kNarrowPhase_new + the set expansion + kFindClosestFace,
 * GPU_Functionality.cs:539-616): the impact list is the one
 * icf_broad_phase(ctx, pad) followed by icf_narrow_phase(ctx, -1, NULL, ...)
 * gives, found by one query per surface node in a grid of the surface
 * elements.  The pair list and the narrow-phase masks are left as they were.
 * Requires CollisionScheme != 0 (with 0 the list is empty). */
int icf_detect_contacts(icf_ctx *ctx, double pad, int *n_impacts);
int icf_get_pairs(icf_ctx *ctx, int capacity, int *pairs);
/* impacts[n*4] = (node, face vertex 0, 1, 2), the c_itet rows of :611. */
int icf_get_impacts(icf_ctx *ctx, int capacity, int *impacts);
/* Supply an impact list directly (e.g. one read back with ReadImpacts). */
int icf_set_impacts(icf_ctx *ctx, int n_impacts, const int *impacts);
/* 8-bit inclusion masks of the last icf_narrow_phase call (kNarrowPhase_new
 * output, narrowphase.h:91-154), one per pair. */
int icf_get_narrow_masks(icf_ctx *ctx, int capacity, int *masks);

/* ---- pattern, LinearSystem.CreateStructure :29-43 ------------------------ */
/* Static pattern plus the contact pairs of the current impacts
 * (ImplicitModel3.cs:177-196), columns ascending per row
 * (CSRDictionary.cs:64-97).  Returns N (rows) and nnz (blocks). */
int icf_create_structure(icf_ctx *ctx, int *N, int *nnz);
/* csr_rows[N+1], csr_cols[nnz] (the ia/ja arrays handed to PARDISO). */
int icf_get_structure(icf_ctx *ctx, int *csr_rows, int *csr_cols);
/* Per-unit slot maps in the reference's logical layout (the pcsr part of
 * g_ie_pcsr / g_icz / g_icr, GPU_Functionality.cs:355-368, 388-401,
 * 645-662): kind 0 = elements (20 ints each: 16 slots i*4+j, 4 rows),
 * kind 1 = CZs (42 ints: 36 slots i*6+j, 6 rows), kind 2 = impacts (20). */
int icf_get_pcsr(icf_ctx *ctx, int kind, long long capacity, int *out);

/* ---- assembly, AssembleElemsAndCZs :439-479 + collisionResponse :627-676 */
/* Zero, element, CZ (with tentative damage state and flags) and contact
 * contributions into the device BCSR values and rhs.  Synchronous. */
int icf_assemble(icf_ctx *ctx, double h, icf_counts *counts);
/* Same work, enqueued on the context stream without waiting; counters are
 * read later with icf_read_counts, which first repeats the assembly if its CZ
 * law left a failure test undecided (see nLawExact).  Capturable in a CUDA
 * graph once the pattern is built. */
int icf_assemble_async(icf_ctx *ctx, double h);
/* The assembly runs as a fork/join DAG over three streams, captured once as a
 * CUDA graph (default) and re-captured only when the pattern, parameters,
 * buffers or time step change; enable = 0 launches the kernels directly. */
int icf_set_graph(icf_ctx *ctx, int enable);
int icf_read_counts(icf_ctx *ctx, icf_counts *counts);
/* Per-kernel device times of the assembly.  No counterpart in the reference
 * (icFlow times whole steps on the host).  Runs `reps` assemblies without the
 * graph, every kernel on the context stream in the graph's order with an event
 * after it, and returns per kernel its name, its algorithmic bytes per launch
 * (every input and output item counted once) and its mean device time.  The
 * last entry, k_cz_hist, is the refresh of the CZ history-axis cache, which
 * runs once per committed damage state (before the next assembly), not once
 * per assembly.  The outputs of the last run are those of icf_assemble.
 * Synchronous. */
#define ICF_MAX_KERNELS 16
typedef struct icf_kernel_times {
  int n_kernels;               /* kernels one assembly launches */
  char name[ICF_MAX_KERNELS][32];
  long long bytes[ICF_MAX_KERNELS];
  double ms[ICF_MAX_KERNELS];
} icf_kernel_times;
int icf_profile_assembly(icf_ctx *ctx, double h, int reps, icf_kernel_times *out);
/* Launch-variant autotuner.  No counterpart in the reference (its kernels run
 * one thread per unit in blocks of 128, GPU_Functionality.cs:38).  The tet
 * kernel and the two gathers each have several launch variants that compute
 * the same values (registers per thread, codes per iteration, loads through
 * registers or cp.async, lanes per row of the diagonal gather).  icf_autotune
 * times every variant on the current model (`reps` launches each, device
 * events), keeps the fastest of each kind for the following assemblies and
 * reports all timings.  Needs a structure; leaves the outputs of a complete
 * assembly behind.  icf_set_variant pins one variant by index (kind 0 tet,
 * 1 off-diagonal gather, 2 diagonal gather, 4 CZ kernel) or the staging layout (kind 3:
 * 0 per-tet records gathered through contribution codes, the default; 1
 * per-contribution records written at their gather positions and read as
 * streams) or the list split (kind 5, per-tet records only: 0, the default,
 * one list per gather; 1 keeps the units without CZ contributions in lists of
 * their own that run beside the CZ kernel) or the gather scheme (kind 6,
 * per-tet records only: 0, the default, the off-diagonal and diagonal list
 * gathers; 1 one row-tile gather, a CTA per set of rows with the rows' tet
 * records and codes staged in shared memory, built on the host at the first
 * structure that needs it).  The tuner also times whole
 * assemblies with each layout and split first. */
#define ICF_MAX_TUNE 64
typedef struct icf_tune_report {
  int n;                          /* candidates timed */
  char kernel[ICF_MAX_TUNE][16];
  char variant[ICF_MAX_TUNE][32];
  double ms[ICF_MAX_TUNE];        /* mean device time per launch */
  int chosen[ICF_MAX_TUNE];       /* 1 for the variant kept */
} icf_tune_report;
int icf_autotune(icf_ctx *ctx, double h, int reps, icf_tune_report *out);
int icf_set_variant(icf_ctx *ctx, int kind, int variant);
/* Allocation-free assembly.  No counterpart in the reference: icFlow always
 * assembles into buffers its GPU class allocated.  For callers that cannot
 * allocate device memory while they assemble (a host that serves every device
 * byte from its own pre-sized pool, or a loop that must not enter the
 * allocator), this computes the same blocks and rhs as icf_assemble from the
 * caller's device arrays d_un, d_vn, d_an (n_nodes*3 doubles each) into the
 * caller's device arrays d_vals (nnz*9) and d_rhs (N*3), with every temporary
 * held in one 8 MiB static device array that each GPU loading the library keeps
 * until exit.  It calls no cudaMalloc or cudaFree.  Models whose temporaries
 * exceed 8 MiB (80 B/node + 256 B/tet + 384 B/CZ + 1056 B/impact) get
 * ICF_ERR_SIZE.  The context must hold constants, static data and a structure
 * from earlier calls.  The first call on a device looks up the array's device
 * address (make it before any stream capture).  All calls share the array:
 * calls that overlap on the GPU race.  The node forces of
 * icf_transfer_updated_state stay those of the last icf_assemble; the
 * tentative CZ state is that of the last assembly of either kind.
 * Synchronous. */
int icf_assemble_noalloc(icf_ctx *ctx, double h, const double *d_un, const double *d_vn,
                         const double *d_an, double *d_vals, double *d_rhs,
                         icf_counts *counts);

/* ---- results ------------------------------------------------------------- */
/* TransferLinearSystemToHost :481-485: vals[nnz*9], rhs[N*3] (either may be
 * NULL). */
int icf_transfer_linear_system(icf_ctx *ctx, double *vals, double *rhs);
/* TransferUpdatedStateToHost :487-528: commits the tentative CZ state on the
 * device (pmax, tmax <- tentative; failed |= tentatively failed) and copies
 * it back; node_F[n_nodes*3] receives the elastic + contact forces of the
 * last assembly.  Any output may be NULL. */
int icf_transfer_updated_state(icf_ctx *ctx, double *pmax, double *tmax,
                               int *failed, double *avg4, double *node_F);
/* Tentative CZ results of the last assembly without committing:
 * tent[n*2] = pmax_, tmax_; flags[n*3] = contact, damaged, failed;
 * avg4[n*4] = avgDn, avgDt, avgTn, avgTt. */
int icf_get_cz_tentative(icf_ctx *ctx, double *tent, int *flags, double *avg4);
/* The cohesive law alone, on the device, as the assembly's CZ kernel
 * evaluates it at one Gauss point: cohesive_law_thermodynamically_consistent
 * (cz_kernels9/cz_kernels.h:37-174) on the PPR functions (PPR_math.h:2-57).
 * In the reference the law is a __device__ function with no entry point of
 * its own; this one exists so that the device law can be checked case by
 * case.  For n states: committed pmax[i], tmax[i] and openings opn[i], opt[i]
 * -> updated pmax_out[i], tmax_out[i], law[i*5] = Tn, Tt, Dnn, Dtt, Dnt and
 * flags[i*3] = contact, failed, and 1 where a failure test was settled with
 * the reference's rounding (as a repeated assembly settles it).  strength[i*2] = sigma_max, tau_max of each
 * state (deln, delt derived as for icf_set_cz_strength), or NULL for the
 * constants of icf_set_constants.  Host arrays; synchronous. */
int icf_cz_law_eval(icf_ctx *ctx, int n, const double *pmax, const double *tmax,
                    const double *opn, const double *opt, const double *strength,
                    double *pmax_out, double *tmax_out, double *law, int *flags);
int icf_get_device_buffers(icf_ctx *ctx, icf_device_buffers *out);

/* ---- Newmark kinematics on the device, Node.cs:62-97 --------------------- */
/* Committed state u, v, a (n_nodes*3 each). */
int icf_set_node_state(icf_ctx *ctx, int n_nodes, const double *u,
                       const double *v, const double *a);
int icf_get_node_state(icf_ctx *ctx, double *u, double *v, double *a,
                       double *du);
/* du for every node (the Newton increment accumulated so far). */
int icf_set_du(icf_ctx *ctx, int n_nodes, const double *du);
/* InferTentativeValues (Node.cs:89-97) for all nodes, then the device node
 * state used by icf_assemble is updated, as icf_transfer_nodes would. */
int icf_infer_tentative(icf_ctx *ctx, double h);
/* _XtoDU (ImplicitModel3.cs:247-256): du += dx[altId] for active nodes;
 * dx has N*3 entries.  Returns sum(dx^2) in *norm (NormOfDx). */
int icf_add_dx(icf_ctx *ctx, const double *dx, double *norm);
/* The Newton linear solve on the device, replacing LinearSystem.Solve
 * (LinearSystem.cs:48-64, MKL PARDISO on the host, after the D2H of
 * :481-485).  Solves A dx = rhs for the matrix and rhs of the last assembly
 * (A symmetric, stored as its upper blocks, possibly indefinite as PARDISO's
 * mtype -2 allows) by MINRES with a 3x3 block-Jacobi preconditioner (a row
 * whose diagonal block is not positive definite is preconditioned by |S|^-1 of
 * the block's symmetric part S), until the preconditioned residual is at most
 * rel_tol times its initial value.  dx[N*3] (nullable) receives the solution,
 * which also stays on the device for icf_apply_dx.  ICF_ERR_NUMERIC if it does
 * not converge in max_iter iterations, a diagonal block is zero or not finite,
 * or the recurrence breaks down. */
int icf_solve(icf_ctx *ctx, double rel_tol, int max_iter, double *dx, int *iters, double *relres);
/* Sum of squares of the rhs of the last assembly (the Newton residual norm,
 * squared).  No counterpart in the reference, whose convergence test is on
 * the increment (LinearSystem.NormOfDx). */
int icf_residual_norm(icf_ctx *ctx, double *norm2);
/* _XtoDU with the device solution of icf_solve: du += dx for active nodes;
 * *norm = sum(dx^2) (LinearSystem.NormOfDx, LinearSystem.cs:69-74). */
int icf_apply_dx(icf_ctx *ctx, double *norm);
/* AcceptTentativeValues (Node.cs:62-77). */
int icf_accept_tentative(icf_ctx *ctx, double h);

/* ---- learned Newton warm start (no counterpart in the reference) ----------
 * icFlow starts each Newton loop from du = v h (ImplicitModel3.cs:149-156).
 * icf_mlp is a per-node network 15 -> 64 -> 64 -> 3 with GELU, BF16 weights
 * and FP32 accumulation (tensor-core mma), with its own training.  Inputs per
 * node: u, v, a, du of the previous step, du of the step before (15 floats);
 * they are normalised as (x - shift) * scale; the output is in units of
 * out_scale.  norm = {shift[15], scale[15], out_scale[3]}.  Parameters
 * (icf_mlp_param_count floats): W1[64][15] b1[64] W2[64][64] b2[64] W3[3][64]
 * b3[3].  All calls are synchronous; host arrays are row-major per node. */
typedef struct icf_mlp icf_mlp;
int icf_mlp_create(int device, icf_mlp **out);
int icf_mlp_destroy(icf_mlp *m);
const char *icf_mlp_last_error(const icf_mlp *m);
int icf_mlp_param_count(void);
int icf_mlp_set_params(icf_mlp *m, const float *params, const float *norm);
int icf_mlp_get_params(icf_mlp *m, float *params, float *norm);
/* y[n*3] = network(x[n*15]) */
int icf_mlp_forward(icf_mlp *m, int n, const float *x, float *y);
/* the forward's intermediate values for n nodes (host buffers): z1, z2 the
 * float32 pre-activations [n][64], h1, h2 = bf16(GELU(z)) as floats [n][64],
 * y the output [n][3] of icf_mlp_forward; for checking the kernels layer by
 * layer (no reference counterpart) */
int icf_mlp_forward_trace(icf_mlp *m, int n, const float *x, float *z1, float *h1, float *z2, float *h2, float *y);
/* gradient of the mean squared error over n nodes and 3 outputs */
int icf_mlp_grad(icf_mlp *m, int n, const float *x, const float *y, float *grad, float *loss);
/* gradient for a loss the caller defines: dy[n*3] = dL/d(output), so that
 * any loss on the outputs (e.g. the force residual of the predicted
 * increments) trains through the same backward kernels; grad may be NULL
 * (kept on the device for icf_mlp_adam_step) */
int icf_mlp_grad_dy(icf_mlp *m, int n, const float *x, const float *dy, float *grad);
/* one Adam step with grad (NULL: the gradient of the last icf_mlp_grad_dy) */
int icf_mlp_adam_step(icf_mlp *m, const float *grad, float lr);
/* minibatch Adam on the device; epochs over a seeded shuffle; *loss = final
 * mean squared error over all n */
int icf_mlp_train(icf_mlp *m, int n, const float *x, const float *y, int epochs, int batch, float lr,
                  unsigned long long seed, float *loss);

#ifdef __cplusplus
}
#endif
#endif
