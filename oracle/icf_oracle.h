/* icf_oracle.h -- CPU restatement of icFlow's per-Newton-iteration assembly
 * path, used as the CHECKER for the CUDA implementation.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product (icflow_b200/, the C-ABI
 * library) includes, links or calls this code. Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
 *
 * Parity pin: every function here is checked against the reference's own
 * kernel code compiled for the host (oracle/_ref, built by oracle/Makefile
 * from the reference sources read in place) and against the golden fixtures
 * in tests/golden/ that were produced by that build.
 *
 * Layouts are plain arrays-of-structures: node fields are [n][3], unit node
 * lists are [n][4] (tets, impacts) or [n][6] (CZs).  All citations are paths
 * inside the reference project.
 */
#ifndef ICF_ORACLE_H
#define ICF_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Park-Paulino-Roesler constants (cz_kernels9/cz_constants.h:6-14). */
typedef struct orc_ppr {
  double G_fn, G_ft, f_tn, f_tt, alpha, beta, rn, rt;
  double p_m, p_n, deln, delt, pMtn, pMnt, gam_n, gam_t;
} orc_ppr;

/* Model parameters (v3Library/Simulation/DataSheets/ModelPrms.cs). */
typedef struct orc_prms {
  /* inputs, ModelPrms.cs:29-209 */
  double Y, nu, rho, dampingMass, dampingStiffness, gravity;
  double NewmarkBeta, NewmarkGamma;
  double alpha, beta, lambda_n, lambda_t, phi_n, phi_t, sigma_max, tau_max;
  double penaltyK, DistanceEpsilon;
  /* derived, ModelPrms.cs:237-322 and :112-113 */
  double E[36];   /* E[i*6+j] */
  double M[144];  /* M[i*12+j], to be multiplied by the element volume */
  double sf[9];   /* sf[node*3+gp] */
  double B[162];  /* B[(gp*3+coord)*18+dof] */
  orc_ppr ppr;
  double nThreshold, tThreshold;
} orc_prms;

void orc_ppr_derive(orc_ppr *q, double alpha, double beta, double lambda_n,
                    double lambda_t, double phi_n, double phi_t,
                    double sigma_max, double tau_max);
void orc_prms_derive(orc_prms *p);

/* PPR potential derivatives: out = Tn, Tt, Dnn, Dtt, Dnt. */
void orc_ppr_eval(const orc_ppr *q, double dn, double dt, double out[5]);
/* Cohesive law with unload/reload and contact; pmax/tmax updated in place.
 * out = Tn Tt Dnn Dtt Dnt Dtn; flags = contact, failed. */
void orc_cz_law(const orc_ppr *q, double *pmax, double *tmax, double opn,
                double opt, double out[6], int flags[2]);

/* Corotational tet: f[12], Df[144], rest volume. */
void orc_elem_F_Df(const orc_prms *p, const double x0[12], const double un[12],
                   double f[12], double Df[144], double *V);
/* Newmark effective LHS[144] and rhs[12] of one tet (before the scatter). */
void orc_elem_local(const orc_prms *p, double h, const double x0[12],
                    const double un[12], const double vn[12],
                    const double an[12], double lhs[144], double rhs[12]);

/* One CZ before the scatter.  tent = pmax_, tmax_ (max over Gauss points);
 * flags = contact, damaged, failed; avg = avgDn avgDt avgTn avgTt (zero if
 * the CZ failed, as the reference leaves them unwritten). */
void orc_cz_local(const orc_prms *p, const orc_ppr *q, const double x0[18],
                  const double un[18], const double pmax_in[3],
                  const double tmax_in[3], double keff[324], double rhs[18],
                  double tent[2], int flags[3], double avg[4]);

/* Squared point-triangle distance with gradient fd[12] and Hessian sd[144];
 * x = (p, v0, v1, v2). */
double orc_pt(const double x[12], double fd[12], double sd[144], double *s,
              double *t, int *branch);
/* Squared distance node -> triangle with clamped barycentrics. */
double orc_dtn(const double f[9], const double p[3]);
/* 8-bit vertex inclusion mask of two tets, 0 if they share a node. */
int orc_narrow_mask(const double xa[12], const double xb[12], const int na[4],
                    const int nb[4]);
/* Penalty contact of one impact: returns 1 if a response is produced. */
int orc_contact_local(const orc_prms *p, const double x[12], double lhs[144],
                      double rhs[12]);

/* Upper-triangular 3x3-block pattern.  Rows are the alt ids of the active
 * nodes (alt[node] = -1 for anchored nodes).  Static pairs come from the
 * tets and from every CZ in cz_static; dynamic pairs from the impacts.
 * Returns N (the number of rows); fills csr_rows[N+1] and, if csr_cols is
 * non-NULL, csr_cols[nnz] (capacity cap).  *nnz receives the count.
 * Returns -1 on capacity overflow. */
int orc_build_structure(int n_nodes, const int *alt, int n_elem,
                        const int *elem, int n_cz, const int *cz, int n_imp,
                        const int *imp, int *csr_rows, int *csr_cols,
                        int *nnz, long long cap);
int orc_slot(const int *csr_rows, const int *csr_cols, int N, int i, int j);
/* Per-unit slot map: k nodes per unit; out[u*(k*k+k) + i*k + j] = slot of
 * block (i,j) or -1; out[u*(k*k+k) + k*k + i] = rhs row of node i or -1. */
void orc_pcsr(int n_units, int k, const int *unit_nodes, const int *alt,
              const int *csr_rows, const int *csr_cols, int N, int *out);

/* Full assembly, sequential and in unit order (elements, then CZs, then
 * impacts).  vals[nnz*9], rhs[N*3] and nodeF[n_nodes*3] are accumulated
 * (zero them first).  cz_ppr may be NULL (global constants).  Per-CZ outputs:
 * tent[2*c] = pmax_, tmax_; flags[3*c] = contact, damaged, failed;
 * avg[4*c]. */
void orc_assemble(const orc_prms *p, double h, int n_nodes, const double *x0,
                  const double *un, const double *vn, const double *an,
                  const double *xt, int n_elem, const int *elem,
                  const int *elem_pcsr, int n_cz, const int *cz,
                  const int *cz_pcsr, const orc_ppr *cz_ppr,
                  const double *pmax, const double *tmax, int n_imp,
                  const int *imp, const int *imp_pcsr, double *vals,
                  double *rhs, double *nodeF, double *tent, int *flags,
                  double *avg);

/* Narrow phase over surface-element pairs: masks[i]. */
void orc_narrow_phase(int n_pairs, const int *pairs, const int *selem,
                      const double *xt, int *masks);
/* Expands masks into the (node, element) set, sorted ascending by
 * (node, element), and resolves each to its closest adjacent face.
 * adj_off[n_selem+1]/adj_faces list each surface element's adjacent faces in
 * order; faces[3*f] are global node ids.  out[4*i] = p, f0, f1, f2.
 * Returns the impact count, or -1 if cap is exceeded. */
int orc_impacts(int n_pairs, const int *pairs, const int *masks,
                const int *selem, const int *adj_off, const int *adj_faces,
                const int *faces, const double *xt, int *out, int cap);

/* Broad phase of the reference: the element pairs its k-DOP-24 bounding
 * volume hierarchy reports (BVHT.cs:29-77).  Every surface element gets the
 * 24-plane k-DOP of its tentative vertices (kDOP24.cs:69-141); a node's box
 * contains its children's (BVHN.cs:39-161), so the self-collide traversal
 * (BVHN.cs:166-194) lists exactly the unordered leaf pairs whose k-DOPs
 * overlap (kDOP24.cs:84-113), whatever the tree's shape.  out[2*i] < out[2*i+1],
 * pairs ascending.  Returns the pair count, or -1 if cap is exceeded. */
int orc_kdop_pairs(int n_selem, const int *selem, const double *xt, int *out, long long cap);

/* The candidate pairs the device broad phase hands the narrow phase, by a
 * uniform grid on the host: surface elements a < b whose boxes at xt overlap
 * (closed), that share no node and where a vertex of one lies in the other's
 * box; with group != NULL only pairs of different groups.  out[2*i] <
 * out[2*i+1], ascending.  Returns the count, or -1 if cap is exceeded. */
long long orc_candidate_pairs(int n_selem, const int *selem, const int *group, const double *xt,
                              double pad, int *out, long long cap);

/* Newmark predictor (Node.cs:89-97 with :79-87) and commit (Node.cs:62-77). */
void orc_newmark_infer(int n, double h, double beta, double gamma,
                       const double *x0, const double *u, const double *v,
                       const double *a, const double *du, double *un,
                       double *vn, double *an, double *xt);
void orc_newmark_accept(int n, double h, const double *x0, double *u,
                        double *v, double *a, const double *un, double *du,
                        double *xc);

#ifdef __cplusplus
}
#endif
#endif
