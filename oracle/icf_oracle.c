/* icf_oracle.c -- CPU restatement of icFlow's per-Newton-iteration assembly
 * path: the CHECKER for the CUDA implementation.
 *
 * TEST INFRASTRUCTURE ONLY.  The product never links or calls this file; only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg do.
 *
 * Parity pin: checked in tests/ against the reference's kernel sources built
 * for the host (oracle/_ref) and against fixtures in tests/golden/ produced by
 * that build.  Built with -ffp-contract=off so that every product and sum is
 * rounded separately, which makes the results reproducible bit for bit across
 * compilers; the CUDA kernels use the same rounding wherever a comparison
 * (inclusion tests, closest face, Voronoi region) decides an integer output.
 *
 * Citations are paths inside the reference project.
 */
#include "icf_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Model parameters                                                          */
/* ------------------------------------------------------------------------ */

static double macaulay(double a, double b) { return a > b ? a - b : 0.0; }

/* ModelPrms.Recompute / SetComputedVariables PPR part, ModelPrms.cs:79-107
 * and :259-285. */
void orc_ppr_derive(orc_ppr *q, double alpha, double beta, double lambda_n,
                    double lambda_t, double phi_n, double phi_t,
                    double sigma_max, double tau_max) {
  q->alpha = alpha;
  q->beta = beta;
  q->G_fn = phi_n;
  q->G_ft = phi_t;
  q->f_tn = sigma_max;
  q->f_tt = tau_max;
  q->rn = lambda_n;
  q->rt = lambda_t;
  q->pMnt = macaulay(q->G_fn, q->G_ft);
  q->pMtn = macaulay(q->G_ft, q->G_fn);
  const double rn2 = q->rn * q->rn, rt2 = q->rt * q->rt;
  q->p_m = (alpha * (alpha - 1.0) * rn2) / (1.0 - alpha * rn2);
  q->p_n = (beta * (beta - 1.0) * rt2) / (1.0 - beta * rt2);
  if (q->G_fn < q->G_ft) {
    q->gam_n = pow(alpha / q->p_m, q->p_m);
    q->gam_t = -q->G_ft * pow(beta / q->p_n, q->p_n);
  } else {
    q->gam_n = -q->G_fn * pow(alpha / q->p_m, q->p_m);
    q->gam_t = pow(beta / q->p_n, q->p_n);
  }
  q->deln = (q->G_fn / q->f_tn) * alpha * q->rn * pow(1.0 - q->rn, alpha - 1.0) *
            ((alpha / q->p_m) + 1.0) *
            pow((alpha / q->p_m) * q->rn + 1.0, q->p_m - 1.0);
  q->delt = (q->G_ft / q->f_tt) * beta * q->rt * pow(1.0 - q->rt, beta - 1.0) *
            ((beta / q->p_n) + 1.0) *
            pow((beta / q->p_n) * q->rt + 1.0, q->p_n - 1.0);
}

/* ModelPrms.SetComputedVariables, ModelPrms.cs:237-349; thresholds :112-113. */
void orc_prms_derive(orc_prms *p) {
  /* consistent mass pattern: rho/20 on same-component entries, doubled on
   * the diagonal (ModelPrms.cs:239-248) */
  const double mc = p->rho / 20.0;
  for (int r = 0; r < 12; r++)
    for (int c = 0; c < 12; c++)
      p->M[r * 12 + c] = (r % 3 == c % 3) ? (r == c ? 2.0 * mc : mc) : 0.0;

  /* isotropic elasticity with engineering shear strains (ModelPrms.cs:250-257) */
  const double k = p->Y / ((1.0 + p->nu) * (1.0 - 2.0 * p->nu));
  memset(p->E, 0, sizeof p->E);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) p->E[i * 6 + j] = (i == j ? 1.0 - p->nu : p->nu) * k;
  for (int i = 3; i < 6; i++) p->E[i * 6 + i] = (0.5 - p->nu) * k;

  orc_ppr_derive(&p->ppr, p->alpha, p->beta, p->lambda_n, p->lambda_t,
                 p->phi_n, p->phi_t, p->sigma_max, p->tau_max);
  p->nThreshold = p->ppr.deln * p->lambda_n;
  p->tThreshold = p->ppr.delt * p->lambda_t;

  /* three-point rule on the triangle; sf[node][gp] (ModelPrms.cs:288-307) */
  const double g1[3] = {1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0};
  const double g2[3] = {2.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0};
  for (int gp = 0; gp < 3; gp++) {
    p->sf[0 * 3 + gp] = 1.0 - g1[gp] - g2[gp];
    p->sf[1 * 3 + gp] = g1[gp];
    p->sf[2 * 3 + gp] = g2[gp];
  }
  /* opening operator: +sf on the first face's dofs, -sf on the second's
   * (ModelPrms.cs:324-349) */
  memset(p->B, 0, sizeof p->B);
  for (int gp = 0; gp < 3; gp++)
    for (int n = 0; n < 3; n++)
      for (int c = 0; c < 3; c++) {
        p->B[(gp * 3 + c) * 18 + 3 * n + c] = p->sf[n * 3 + gp];
        p->B[(gp * 3 + c) * 18 + 9 + 3 * n + c] = -p->sf[n * 3 + gp];
      }
}

/* ------------------------------------------------------------------------ */
/* PPR potential, cz_kernels9/PPR_math.h:2-57                                */
/* ------------------------------------------------------------------------ */

/* Power factors of one PPR axis at normalised opening x = delta / del:
 *   o_k = (1-x)^(a-k),  s_k = (p/a + x)^(p-k),  k = 0, 1, 2.
 * The five PPR functions below are products of these, grouped left to right
 * in the same order as PPR_math.h so the rounding matches the reference. */
typedef struct { double o0, o1, o2, s0, s1, s2; } ppr_pw;
static ppr_pw ppr_pows(double a, double p, double x) {
  ppr_pw w;
  const double o = 1.0 - x, s = (p / a) + x;
  w.o0 = pow(o, a);
  w.o1 = pow(o, a - 1.0);
  w.o2 = pow(o, a - 2.0);
  w.s0 = pow(s, p);
  w.s1 = pow(s, p - 1.0);
  w.s2 = pow(s, p - 2.0);
  return w;
}

/* Tn_ (PPR_math.h:2-12): (gam_n/deln) * dPhi_n * (gam_t Phi_t + <phi_t-phi_n>) */
static double ppr_Tn(const orc_ppr *q, double dn, double dt) {
  const ppr_pw N = ppr_pows(q->alpha, q->p_m, dn / q->deln);
  const ppr_pw T = ppr_pows(q->beta, q->p_n, dt / q->delt);
  const double d1 = (q->p_m * N.o0 * N.s1) - (q->alpha * N.o1 * N.s0);
  const double ft = q->gam_t * T.o0 * T.s0 + q->pMtn;
  return (q->gam_n / q->deln) * d1 * ft;
}
/* Tt_ (PPR_math.h:14-24) */
static double ppr_Tt(const orc_ppr *q, double dn, double dt) {
  const ppr_pw N = ppr_pows(q->alpha, q->p_m, dn / q->deln);
  const ppr_pw T = ppr_pows(q->beta, q->p_n, dt / q->delt);
  const double d1 = q->p_n * T.o0 * T.s1 - q->beta * T.o1 * T.s0;
  const double fn = q->gam_n * N.o0 * N.s0 + q->pMnt;
  return (q->gam_t / q->delt) * d1 * fn;
}
/* Dnn_ (PPR_math.h:26-35) */
static double ppr_Dnn(const orc_ppr *q, double dn, double dt) {
  const ppr_pw N = ppr_pows(q->alpha, q->p_m, dn / q->deln);
  const ppr_pw T = ppr_pows(q->beta, q->p_n, dt / q->delt);
  const double a = q->alpha, p = q->p_m;
  const double e1 = (p * p - p) * N.o0 * N.s2;
  const double e2 = (a * a - a) * N.o2 * N.s0;
  const double e3 = 2.0 * a * p * N.o1 * N.s1;
  const double ft = q->gam_t * T.o0 * T.s0 + q->pMtn;
  return (q->gam_n / (q->deln * q->deln)) * (e1 + e2 - e3) * ft;
}
/* Dtt_ (PPR_math.h:37-46) */
static double ppr_Dtt(const orc_ppr *q, double dn, double dt) {
  const ppr_pw N = ppr_pows(q->alpha, q->p_m, dn / q->deln);
  const ppr_pw T = ppr_pows(q->beta, q->p_n, dt / q->delt);
  const double b = q->beta, p = q->p_n;
  const double e1 = (p * p - p) * T.o0 * T.s2;
  const double e2 = (b * b - b) * T.o2 * T.s0;
  const double e3 = 2.0 * b * p * T.o1 * T.s1;
  const double fn = q->gam_n * N.o0 * N.s0 + q->pMnt;
  return (q->gam_t / (q->delt * q->delt)) * (e1 + e2 - e3) * fn;
}
/* Dnt_ (PPR_math.h:48-57) */
static double ppr_Dnt(const orc_ppr *q, double dn, double dt) {
  const ppr_pw N = ppr_pows(q->alpha, q->p_m, dn / q->deln);
  const ppr_pw T = ppr_pows(q->beta, q->p_n, dt / q->delt);
  const double dN = q->p_m * N.o0 * N.s1 - q->alpha * N.o1 * N.s0;
  const double dT = q->p_n * T.o0 * T.s1 - q->beta * T.o1 * T.s0;
  return (q->gam_n * q->gam_t / (q->deln * q->delt)) * dN * dT;
}

void orc_ppr_eval(const orc_ppr *q, double dn, double dt, double out[5]) {
  out[0] = ppr_Tn(q, dn, dt);
  out[1] = ppr_Tt(q, dn, dt);
  out[2] = ppr_Dnn(q, dn, dt);
  out[3] = ppr_Dtt(q, dn, dt);
  out[4] = ppr_Dnt(q, dn, dt);
}

/* cohesive_law_thermodynamically_consistent, cz_kernels.h:37-174.
 * The branch structure is the algorithm and is kept as in the reference. */
void orc_cz_law(const orc_ppr *q, double *pmax, double *tmax, double opn,
                double opt, double out[6], int flags[2]) {
  double Tn = 0, Tt = 0, Dnn = 0, Dtt = 0, Dnt = 0;
  int contact = flags[0], failed = flags[1];
  if (opn > q->deln || opt > q->delt) { /* :40-42 */
    failed = 1;
    goto done;
  }
  contact = (opn < 0);
  {
    const double eps_neg = -1e-9;                 /* :44 */
    const double thr_t = q->f_tt * 0.05;          /* :45-46 */
    const double thr_n = q->f_tn * 0.05;          /* :47 */
    if (contact) {                                /* :49-87 */
      Dnt = 0;
      if (*pmax != 0) {
        const double peak = ppr_Tn(q, *pmax, *tmax);
        Tn = peak * opn / *pmax;
        Dnn = peak / *pmax;
      } else {
        Dnn = ppr_Dnn(q, 0, *tmax);
        Tn = Dnn * opn;
      }
      Tt = ppr_Tt(q, 0, opt);
      if (Tt >= eps_neg && !(opt > q->delt * q->rt / 5 && Tt < thr_t)) {
        if (opt >= *tmax) {
          *tmax = opt;
          Dtt = ppr_Dtt(q, 0, opt);
        } else {
          const double peak = ppr_Tt(q, 0, *tmax);
          Tt = peak * opt / *tmax;
          Dtt = peak / *tmax;
        }
      } else {
        Tt = Dtt = Dnt = 0;
        Tn = Dnn = 0;
        failed = 1;
      }
    } else {                                      /* :88-172 */
      Tt = ppr_Tt(q, opn, opt);
      Tn = ppr_Tn(q, opn, opt);
      if (Tt >= eps_neg && Tn >= eps_neg &&
          !(opt > q->delt * q->rt / 5 && Tt < thr_t) &&
          !(opn > q->deln * q->rn / 5 && Tn < thr_n)) {
        const int tsoft = (opt >= *tmax), nsoft = (opn >= *pmax);
        if (tsoft && nsoft) {                     /* :100-108 */
          *tmax = opt;
          *pmax = opn;
          Dnn = ppr_Dnn(q, opn, opt);
          Dnt = ppr_Dnt(q, opn, opt);
          Dtt = ppr_Dtt(q, opn, opt);
        } else if (tsoft && !nsoft) {             /* :109-124 */
          Dnt = 0;
          if (*pmax != 0) {
            const double peak = ppr_Tn(q, *pmax, *tmax);
            Tn = peak * opn / *pmax;
            Dnn = peak / *pmax;
          } else {
            Tn = 0;
            Dnn = ppr_Dnn(q, 0, *tmax);
          }
          *tmax = opt;
          Tt = ppr_Tt(q, *pmax, opt);
          Dtt = ppr_Dtt(q, *pmax, opt);
        } else if (!tsoft && nsoft) {             /* :125-141 */
          Dnt = 0;
          if (*tmax != 0) {
            const double peak = ppr_Tt(q, *pmax, *tmax);
            Tt = peak * opt / *tmax;
            Dtt = peak / *tmax;
          } else {
            Tt = 0;
            Dtt = ppr_Dtt(q, *pmax, 0);
          }
          *pmax = opn;
          Tn = ppr_Tn(q, *pmax, *tmax);
          Dnn = ppr_Dnn(q, *pmax, *tmax);
        } else {                                  /* :142-164 */
          Dnt = 0;
          const double peakN = ppr_Tn(q, *pmax, *tmax);
          if (*pmax != 0) {
            Tn = peakN * opn / *pmax;
            Dnn = peakN / *pmax;
          } else {
            Tn = 0;
            Dnn = ppr_Dnn(q, 0, *tmax);
          }
          if (*tmax != 0) {
            const double peakT = ppr_Tt(q, *pmax, *tmax);
            Tt = peakT * opt / *tmax;
            Dtt = peakT / *tmax;
          } else {
            Tt = 0;
            Dtt = ppr_Dtt(q, *pmax, 0);
          }
        }
      } else {                                    /* :167-171 */
        failed = 1;
        Tn = Tt = Dnn = Dtt = Dnt = 0;
      }
    }
  }
done:
  out[0] = Tn;
  out[1] = Tt;
  out[2] = Dnn;
  out[3] = Dtt;
  out[4] = Dnt;
  out[5] = Dnt; /* Dtn = Dnt, :173 */
  flags[0] = contact;
  flags[1] = failed;
}

/* ------------------------------------------------------------------------ */
/* Corotational tetrahedron, elem_kernels9/element_kernels2.h                 */
/* ------------------------------------------------------------------------ */

/* Orthonormal frame from three points, fastRotationMatrix
 * (elem_kernels9/matrix_math1.h:32-71): column 0 = unit(p1-p0), column 1 =
 * unit((p1-p0) x (p2-p0)), column 2 = unit(column 1 x column 0). */
static void frame3(const double *p0, const double *p1, const double *p2,
                   double R[3][3]) {
  double d[3], w[3], c[3];
  for (int k = 0; k < 3; k++) {
    d[k] = p1[k] - p0[k];
    w[k] = p2[k] - p0[k];
  }
  double m = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  for (int k = 0; k < 3; k++) R[k][0] = d[k] / m;
  c[0] = -d[2] * w[1] + d[1] * w[2];
  c[1] = d[2] * w[0] - d[0] * w[2];
  c[2] = -d[1] * w[0] + d[0] * w[1];
  m = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
  for (int k = 0; k < 3; k++) R[k][1] = c[k] / m;
  R[0][2] = R[1][1] * R[2][0] - R[1][0] * R[2][1];
  R[1][2] = -R[0][1] * R[2][0] + R[0][0] * R[2][1];
  R[2][2] = R[0][1] * R[1][0] - R[0][0] * R[1][1];
  m = sqrt(R[0][2] * R[0][2] + R[1][2] * R[1][2] + R[2][2] * R[2][2]);
  for (int k = 0; k < 3; k++) R[k][2] /= m;
}

/* F_and_Df_Corotational, element_kernels2.h:19-159:
 *   K = V B^T E B, R = R1 R0^T, f = R K (R^T xc - x0), Df = R K R^T. */
void orc_elem_F_Df(const orc_prms *p, const double x0[12], const double un[12],
                   double f[12], double Df[144], double *Vout) {
  double xc[12];
  for (int i = 0; i < 12; i++) xc[i] = x0[i] + un[i];

  /* difference of coordinate c between nodes i and j (1-based) */
#define DX(c, i, j) (x0[3 * ((i)-1) + (c)] - x0[3 * ((j)-1) + (c)])
  const double Jdet =
      DX(0, 2, 1) * (DX(1, 2, 3) * DX(2, 3, 4) - DX(1, 3, 4) * DX(2, 2, 3)) +
      DX(0, 3, 2) * (DX(1, 3, 4) * DX(2, 1, 2) - DX(1, 1, 2) * DX(2, 3, 4)) +
      DX(0, 4, 3) * (DX(1, 1, 2) * DX(2, 2, 3) - DX(1, 2, 3) * DX(2, 1, 2));
  const double V = Jdet / 6.;

  /* shape-function gradients by cofactors (:50-57); node n uses the two
   * edges (P,Q) and (S,T) listed below */
  static const int PQST[4][4] = {{4, 2, 3, 2}, {3, 1, 4, 3}, {2, 4, 1, 4}, {1, 3, 2, 1}};
  double g[4][3];
  for (int n = 0; n < 4; n++) {
    const int P = PQST[n][0], Q = PQST[n][1], S = PQST[n][2], T = PQST[n][3];
    g[n][0] = (DX(1, P, Q) * DX(2, S, T) - DX(1, S, T) * DX(2, P, Q)) / Jdet;
    g[n][1] = (DX(0, S, T) * DX(2, P, Q) - DX(0, P, Q) * DX(2, S, T)) / Jdet;
    g[n][2] = (DX(0, P, Q) * DX(1, S, T) - DX(0, S, T) * DX(1, P, Q)) / Jdet;
  }
#undef DX

  /* strain-displacement matrix, engineering shear order xy, yz, zx (:59-65) */
  double B[6][12];
  memset(B, 0, sizeof B);
  for (int n = 0; n < 4; n++) {
    const double a = g[n][0], b = g[n][1], c = g[n][2];
    B[0][3 * n + 0] = a;
    B[1][3 * n + 1] = b;
    B[2][3 * n + 2] = c;
    B[3][3 * n + 0] = b; B[3][3 * n + 1] = a;
    B[4][3 * n + 1] = c; B[4][3 * n + 2] = b;
    B[5][3 * n + 0] = c; B[5][3 * n + 2] = a;
  }
  /* K = B^T E B V (:67-76) */
  double BtE[12][6], K[12][12];
  for (int r = 0; r < 12; r++)
    for (int c = 0; c < 6; c++) {
      double s = 0;
      for (int i = 0; i < 6; i++) s += B[i][r] * p->E[i * 6 + c];
      BtE[r][c] = s;
    }
  for (int r = 0; r < 12; r++)
    for (int c = 0; c < 12; c++) {
      double s = 0;
      for (int i = 0; i < 6; i++) s += BtE[r][i] * B[i][c] * V;
      K[r][c] = s;
    }

  /* rotation from rest frame to current frame (:78-104) */
  double R0[3][3], R1[3][3], R[3][3];
  frame3(x0, x0 + 3, x0 + 6, R0);
  frame3(xc, xc + 3, xc + 6, R1);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      R[i][j] = R1[i][0] * R0[j][0] + R1[i][1] * R0[j][1] + R1[i][2] * R0[j][2];

  /* RK and R K R^T per 3x3 block (:106-125) */
  double RK[12][12], RKRt[12][12];
  for (int bi = 0; bi < 4; bi++)
    for (int bj = 0; bj < 4; bj++) {
      for (int k = 0; k < 3; k++)
        for (int l = 0; l < 3; l++) {
          double s = 0;
          for (int m = 0; m < 3; m++) s += R[k][m] * K[3 * bi + m][3 * bj + l];
          RK[3 * bi + k][3 * bj + l] = s;
        }
      for (int k = 0; k < 3; k++)
        for (int l = 0; l < 3; l++) {
          double s = 0;
          for (int m = 0; m < 3; m++) s += RK[3 * bi + k][3 * bj + m] * R[l][m];
          RKRt[3 * bi + k][3 * bj + l] = s;
        }
    }

  /* xr = R^T xc - x0 (:128-150) */
  double xr[12];
  for (int n = 0; n < 4; n++)
    for (int k = 0; k < 3; k++)
      xr[3 * n + k] = xc[3 * n + 0] * R[0][k] + xc[3 * n + 1] * R[1][k] +
                      xc[3 * n + 2] * R[2][k];
  for (int i = 0; i < 12; i++) xr[i] -= x0[i];

  /* f = RK xr, Df = R K R^T (:154-158) */
  for (int i = 0; i < 12; i++) {
    double s = 0;
    for (int j = 0; j < 12; j++) {
      s += RK[i][j] * xr[j];
      Df[i * 12 + j] = RKRt[i][j];
    }
    f[i] = s;
  }
  *Vout = V;
}

/* kelElementElasticityForce before the scatter, element_kernels2.h:222-251:
 *   rhs = g - f - (M V dm + Df ds) vn - M V an
 *   LHS = Df (1 + ds gamma / (h beta)) + M V (1/h^2 + dm gamma / h) / beta */
void orc_elem_local(const orc_prms *p, double h, const double x0[12],
                    const double un[12], const double vn[12],
                    const double an[12], double lhs[144], double rhs[12]) {
  double f[12], Df[144], V;
  orc_elem_F_Df(p, x0, un, f, Df, &V);
  const double gnode = p->gravity * p->rho * V / 4;
  for (int i = 0; i < 12; i++) rhs[i] = (i % 3 == 2) ? gnode : 0.0;
  const double massCoeff =
      V * (1.0 / (h * h) + p->dampingMass * p->NewmarkGamma / h) / p->NewmarkBeta;
  const double stiffCoeff =
      1.0 + p->dampingStiffness * p->NewmarkGamma / (h * p->NewmarkBeta);
  for (int i = 0; i < 12; i++) {
    rhs[i] -= f[i];
    for (int j = 0; j < 12; j++) {
      const double Mij = p->M[i * 12 + j];
      rhs[i] -= (Mij * V * p->dampingMass + Df[i * 12 + j] * p->dampingStiffness) * vn[j] +
                (Mij * V * an[j]);
      lhs[i * 12 + j] = Df[i * 12 + j] * stiffCoeff + Mij * massCoeff;
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Cohesive zone, cz_kernels9/cz_kernels.h:210-434                            */
/* ------------------------------------------------------------------------ */

/* CZRotationMatrix, cz_kernels9/matrix_math.h:15-68: rows are unit(e1),
 * unit(n x e1), unit(n) with e1 = x1 - x0, n = e1 x (x0 - x2); aJ = |n| / 2. */
static void cz_frame(const double *m0, const double *m1, const double *m2,
                     double R[3][3], double *aJ) {
  double p1[3], p2[3], n[3], r[3];
  for (int k = 0; k < 3; k++) {
    p1[k] = m1[k] - m0[k];
    p2[k] = m0[k] - m2[k];
  }
  const double l1 = sqrt(p1[0] * p1[0] + p1[1] * p1[1] + p1[2] * p1[2]);
  for (int k = 0; k < 3; k++) R[0][k] = p1[k] / l1;
  n[0] = -p1[2] * p2[1] + p1[1] * p2[2];
  n[1] = p1[2] * p2[0] - p1[0] * p2[2];
  n[2] = -p1[1] * p2[0] + p1[0] * p2[1];
  double ln = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  *aJ = ln / 2;
  for (int k = 0; k < 3; k++) {
    n[k] /= ln;
    R[2][k] = n[k];
    p1[k] /= l1;
  }
  r[0] = -n[2] * p1[1] + n[1] * p1[2];
  r[1] = n[2] * p1[0] - n[0] * p1[2];
  r[2] = -n[1] * p1[0] + n[0] * p1[1];
  ln = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
  for (int k = 0; k < 3; k++) R[1][k] = r[k] / ln;
}

void orc_cz_local(const orc_prms *p, const orc_ppr *q, const double x0[18],
                  const double un[18], const double pmax_in[3],
                  const double tmax_in[3], double keff[324], double rhs[18],
                  double tent[2], int flags[3], double avg[4]) {
  double xc[18], xr[18], pmax[3], tmax[3];
  for (int i = 0; i < 18; i++) xc[i] = x0[i] + un[i];
  for (int i = 0; i < 3; i++) {
    pmax[i] = pmax_in[i];
    tmax[i] = tmax_in[i];
  }
  /* mid-plane of the two faces and its frame (:243-256) */
  double mp[9], R[3][3], aJ;
  for (int i = 0; i < 9; i++) mp[i] = (xc[i] + xc[i + 9]) * 0.5;
  cz_frame(mp, mp + 3, mp + 6, R, &aJ);
  /* local coordinates xr = R xc (:259-266) */
  for (int n = 0; n < 6; n++)
    for (int k = 0; k < 3; k++)
      xr[3 * n + k] = xc[3 * n + 0] * R[k][0] + xc[3 * n + 1] * R[k][1] +
                      xc[3 * n + 2] * R[k][2];

  memset(keff, 0, 324 * sizeof(double));
  memset(rhs, 0, 18 * sizeof(double));
  int gp_contact[3] = {0, 0, 0}, gp_failed[3] = {0, 0, 0};
  double aDn = 0, aDt = 0, aTn = 0, aTt = 0;
  const double w = 1.0 / 3.0; /* Gauss weight (:344) */

  for (int gp = 0; gp < 3; gp++) {
    /* opening at the Gauss point (:281-290) */
    double o[3] = {0, 0, 0};
    for (int n = 0; n < 3; n++)
      for (int k = 0; k < 3; k++)
        o[k] += (xr[3 * n + k] - xr[3 * n + 9 + k]) * p->sf[n * 3 + gp];
    const double opn = o[2];
    const double opt = sqrt(o[0] * o[0] + o[1] * o[1]);

    double law[6];
    int fl[2] = {gp_contact[gp], gp_failed[gp]};
    orc_cz_law(q, &pmax[gp], &tmax[gp], opn, opt, law, fl);
    gp_contact[gp] = fl[0];
    gp_failed[gp] = fl[1];
    const double Tn = law[0], Tt = law[1], Dnn = law[2], Dtt = law[3],
                 Dnt = law[4], Dtn = law[5];
    aDn += opn / 3;
    aDt += opt / 3;
    aTn += Tn / 3;
    aTt += Tt / 3;

    /* traction and its tangent in the local frame (:301-340) */
    double T[3] = {0, 0, 0}, Td[3][3];
    memset(Td, 0, sizeof Td);
    if (opt < 1e-20) {
      T[2] = Tn;
      Td[0][0] = Dtt;
      Td[1][1] = Dtt;
      Td[2][2] = Dnn;
      Td[2][0] = Dtn;
      Td[0][2] = Dnt;
      Td[2][1] = Dtn;
      Td[1][2] = Dnt;
    } else {
      T[0] = Tt * o[0] / opt;
      T[1] = Tt * o[1] / opt;
      T[2] = Tn;
      const double opt2 = opt * opt, opt3 = opt2 * opt;
      const double u00 = o[0] * o[0], u10 = o[1] * o[0], u11 = o[1] * o[1];
      Td[0][0] = Dtt * u00 / opt2 + Tt * u11 / opt3;
      Td[1][1] = Dtt * u11 / opt2 + Tt * u00 / opt3;
      Td[2][2] = Dnn;
      Td[1][0] = Td[0][1] = Dtt * u10 / opt2 - Tt * u10 / opt3;
      Td[2][0] = Dtn * o[0] / opt;
      Td[0][2] = Dnt * o[0] / opt;
      Td[2][1] = Dtn * o[1] / opt;
      Td[1][2] = Dnt * o[1] / opt;
    }

    const double *Bg = p->B + gp * 54; /* B[gp][coord][dof] */
    /* rhs -= R^T B^T T w aJ (:343-364) */
    double BtT[18];
    for (int i = 0; i < 18; i++) {
      double s = 0;
      for (int j = 0; j < 3; j++) s += Bg[j * 18 + i] * T[j];
      BtT[i] = s * -(w * aJ);
    }
    for (int n = 0; n < 6; n++)
      for (int k = 0; k < 3; k++)
        rhs[3 * n + k] += BtT[3 * n + 0] * R[0][k] + BtT[3 * n + 1] * R[1][k] +
                          BtT[3 * n + 2] * R[2][k];

    /* Keff += R^T (B^T Td B w aJ) R per 3x3 block (:366-401) */
    double BtTd[18][3], BtTdB[18][18];
    for (int r = 0; r < 18; r++)
      for (int c = 0; c < 3; c++) {
        double s = 0;
        for (int k = 0; k < 3; k++) s += Bg[k * 18 + r] * Td[k][c];
        BtTd[r][c] = s * (w * aJ);
      }
    for (int r = 0; r < 18; r++)
      for (int c = 0; c < 18; c++) {
        double s = 0;
        for (int k = 0; k < 3; k++) s += BtTd[r][k] * Bg[k * 18 + c];
        BtTdB[r][c] = s;
      }
    for (int bi = 0; bi < 6; bi++)
      for (int bj = 0; bj < 6; bj++) {
        double Tm[3][3];
        for (int k = 0; k < 3; k++)
          for (int l = 0; l < 3; l++) {
            double s = 0;
            for (int m = 0; m < 3; m++) s += R[m][k] * BtTdB[3 * bi + m][3 * bj + l];
            Tm[k][l] = s;
          }
        for (int k = 0; k < 3; k++)
          for (int l = 0; l < 3; l++)
            for (int m = 0; m < 3; m++)
              keff[(3 * bi + k) * 18 + 3 * bj + l] += Tm[k][m] * R[m][l];
      }
  }

  /* damage state (:404-422) */
  double pm = pmax[0], tm = tmax[0];
  for (int i = 1; i < 3; i++) {
    if (pmax[i] > pm) pm = pmax[i];
    if (tmax[i] > tm) tm = tmax[i];
  }
  int damaged = 0;
  for (int i = 0; i < 3; i++)
    if (pmax[i] >= q->deln * q->rn || tmax[i] >= q->delt * q->rt) damaged = 1;
  const int failed = gp_failed[0] || gp_failed[1] || gp_failed[2];
  const int contact = gp_contact[0] || gp_contact[1] || gp_contact[2];
  tent[0] = pm;
  tent[1] = tm;
  flags[0] = contact;
  flags[1] = failed ? 0 : damaged;
  flags[2] = failed;
  if (failed) {
    avg[0] = avg[1] = avg[2] = avg[3] = 0;
  } else {
    avg[0] = aDn;
    avg[1] = aDt;
    avg[2] = aTn;
    avg[3] = aTt;
  }
}

/* ------------------------------------------------------------------------ */
/* Point-triangle distance and derivatives, collision_kernels9/point_triange_v2.h */
/* ------------------------------------------------------------------------ */

/* Squared distance between points a and b of x[12] with gradient and Hessian
 * (vertex_vertex_distance_and_derivs_12, :115-150). */
static double pt_vv(const double x[12], int ia, int ib, double fd[12],
                    double sd[144]) {
  double dsq = 0;
  for (int k = 0; k < 3; k++) {
    const double d = x[3 * ia + k] - x[3 * ib + k];
    fd[3 * ia + k] = 2 * d;
    fd[3 * ib + k] = -(2 * d);
    sd[(3 * ia + k) * 12 + 3 * ia + k] = 2;
    sd[(3 * ib + k) * 12 + 3 * ib + k] = 2;
    sd[(3 * ia + k) * 12 + 3 * ib + k] = -2;
    sd[(3 * ib + k) * 12 + 3 * ia + k] = -2;
    dsq += d * d;
  }
  return dsq;
}

/* Squared distance from y[0..2] to the line through y[3..5], y[6..8] with
 * derivatives over the 9 coordinates (vertex_edge_distance_and_derivs,
 * :152-232).  With e = q2 - q1 and r = q1 - p:
 *   dist^2 = |r|^2 - (r.e)^2 / |e|^2,
 * differentiated as f1 - g / f2 with f1 = |r|^2, g = (r.e)^2, f2 = |e|^2.
 * The returned value is evaluated directly from the foot point. */
static double pt_line(const double y[9], double fd[9], double sd[81]) {
  const double *P = y, *Q1 = y + 3, *Q2 = y + 6;
  double el2 = 0, rde = 0;
  for (int k = 0; k < 3; k++) {
    el2 += (Q2[k] - Q1[k]) * (Q2[k] - Q1[k]);
    rde += (Q1[k] - P[k]) * (Q2[k] - Q1[k]);
  }
  const double t = -rde / el2, u = 1 - t;
  double dist2 = 0;
  for (int k = 0; k < 3; k++) {
    const double d = P[k] - u * Q1[k] - t * Q2[k];
    dist2 += d * d;
  }

  /* sp = (q1 - p).(q2 - q1) with its derivatives; g = sp^2 */
  double sp = 0, spd[9], spdd[81];
  memset(spdd, 0, sizeof spdd);
  for (int k = 0; k < 3; k++) {
    spd[k] = Q1[k] - Q2[k];
    spd[3 + k] = P[k] - 2 * Q1[k] + Q2[k];
    spd[6 + k] = Q1[k] - P[k];
    spdd[(3 + k) * 9 + 3 + k] = -2;
    spdd[k * 9 + 6 + k] = spdd[(6 + k) * 9 + k] = -1;
    spdd[k * 9 + 3 + k] = spdd[(3 + k) * 9 + k] = 1;
    spdd[(6 + k) * 9 + 3 + k] = spdd[(3 + k) * 9 + 6 + k] = 1;
    sp += (Q1[k] - P[k]) * (Q2[k] - Q1[k]);
  }
  double g = sp * sp, gd[9], gdd[81];
  for (int i = 0; i < 9; i++) {
    gd[i] = 2 * sp * spd[i];
    for (int j = 0; j < 9; j++) gdd[i * 9 + j] = 2 * (spd[i] * spd[j] + sp * spdd[i * 9 + j]);
  }
  /* f1 = |q1 - p|^2 and f2 = |q2 - q1|^2 with their derivatives */
  double f1 = 0, f1d[9] = {0}, f1dd[81], f2 = 0, f2d[9] = {0}, f2dd[81];
  memset(f1dd, 0, sizeof f1dd);
  memset(f2dd, 0, sizeof f2dd);
  for (int k = 0; k < 3; k++) {
    const double a = Q1[k] - P[k], b = Q2[k] - Q1[k];
    f1 += a * a;
    f2 += b * b;
    f1d[3 + k] = 2 * a;
    f1d[k] = -(2 * a);
    f2d[6 + k] = 2 * b;
    f2d[3 + k] = -(2 * b);
    f1dd[(3 + k) * 9 + 3 + k] = f1dd[k * 9 + k] = 2;
    f1dd[(3 + k) * 9 + k] = f1dd[k * 9 + 3 + k] = -2;
    f2dd[(6 + k) * 9 + 6 + k] = f2dd[(3 + k) * 9 + 3 + k] = 2;
    f2dd[(6 + k) * 9 + 3 + k] = f2dd[(3 + k) * 9 + 6 + k] = -2;
  }
  (void)f1;
  const double f2sq = f2 * f2, f2cu = f2sq * f2;
  for (int i = 0; i < 9; i++) {
    fd[i] = f1d[i] + (g * f2d[i] - f2 * gd[i]) / f2sq;
    for (int j = 0; j < 9; j++) {
      const double t1 = -2 * g * f2d[i] * f2d[j] / f2cu;
      const double t2 = (gd[i] * f2d[j] + gd[j] * f2d[i]) / f2sq;
      const double t3 = f1dd[i * 9 + j];
      const double t4 = g * f2dd[i * 9 + j] / f2sq;
      const double t5 = -gdd[i * 9 + j] / f2;
      sd[i * 9 + j] = t1 + t2 + t3 + t4 + t5;
    }
  }
  return dist2;
}

/* Point x[0..2] against the edge between points ia and ib of x[12]; the
 * nearer endpoint is taken as the line origin (ties keep ia)
 * (vertex_edge_distance_and_derivs_12, :237-294). */
static double pt_ve(const double x[12], int ia, int ib, double fd[12],
                    double sd[144]) {
  double da = 0, db = 0;
  for (int k = 0; k < 3; k++) {
    da += (x[k] - x[3 * ia + k]) * (x[k] - x[3 * ia + k]);
    db += (x[k] - x[3 * ib + k]) * (x[k] - x[3 * ib + k]);
  }
  if (da > db) {
    const int s = ia;
    ia = ib;
    ib = s;
  }
  double y[9], yd[9], ydd[81];
  const int blk[3] = {0, ia, ib};
  for (int b = 0; b < 3; b++)
    for (int k = 0; k < 3; k++) y[3 * b + k] = x[3 * blk[b] + k];
  const double r = pt_line(y, yd, ydd);
  for (int bi = 0; bi < 3; bi++)
    for (int k = 0; k < 3; k++) {
      fd[3 * blk[bi] + k] = yd[3 * bi + k];
      for (int bj = 0; bj < 3; bj++)
        for (int l = 0; l < 3; l++)
          sd[(3 * blk[bi] + k) * 12 + 3 * blk[bj] + l] = ydd[(3 * bi + k) * 9 + 3 * bj + l];
    }
  return r;
}

/* A "selector" maps x[12] to a 3-vector as sp*x[block p] + sn*x[block n]
 * (blocks: 0 = point, 1..3 = triangle vertices). */
typedef struct { int bp, bn; } selector;
/* Hessian of the bilinear form (A x).(C x) in 4x4 block form (each block a
 * multiple of the 3x3 identity) and its gradient. */
static void bilinear(selector A, selector C, const double ax[3],
                     const double cx[3], double grad[12], double H4[4][4]) {
  memset(grad, 0, 12 * sizeof(double));
  memset(H4, 0, 16 * sizeof(double));
  for (int k = 0; k < 3; k++) {
    grad[3 * A.bp + k] += cx[k];
    grad[3 * A.bn + k] -= cx[k];
    grad[3 * C.bp + k] += ax[k];
    grad[3 * C.bn + k] -= ax[k];
  }
  const int ab[2] = {A.bp, A.bn}, cb[2] = {C.bp, C.bn};
  const double sg[2] = {1.0, -1.0};
  for (int i = 0; i < 2; i++)
    for (int j = 0; j < 2; j++) {
      H4[ab[i]][cb[j]] += sg[i] * sg[j];
      H4[cb[j]][ab[i]] += sg[i] * sg[j];
    }
}

/* Interior case: squared distance to the plane of the triangle through the
 * barycentric foot point, differentiated through s(x), t(x)
 * (point_plane_distance, :449-582).  With e0 = v1 - v0, e1 = v2 - v0,
 * w = v0 - p and a = e0.e0, b = e0.e1, c = e1.e1, d = e0.w, e = e1.w:
 *   s = (b e - c d) / det, t = (b d - a e) / det, det = a c - b^2,
 *   q = s v1 + t v2 + (1 - s - t) v0 - p, dist^2 = |q|^2. */
static double pt_plane(const double x[12], double fd[12], double sd[144]) {
  const double *P = x, *V0 = x + 3, *V1 = x + 6, *V2 = x + 9;
  double e0[3], e1[3], w[3];
  for (int k = 0; k < 3; k++) {
    e0[k] = -V0[k] + V1[k];
    e1[k] = -V0[k] + V2[k];
    w[k] = -P[k] + V0[k];
  }
  /* b, c and e are summed over y, z, x and a, d over x, y, z, the order in
   * which point_triange_v2.h:605-610 writes them */
  const double a = e0[0] * e0[0] + e0[1] * e0[1] + e0[2] * e0[2];
  const double b = e1[1] * e0[1] + e1[2] * e0[2] + e0[0] * e1[0];
  const double c = e1[1] * e1[1] + e1[2] * e1[2] + e1[0] * e1[0];
  const double d = w[0] * e0[0] + w[1] * e0[1] + w[2] * e0[2];
  const double e = e1[1] * w[1] + e1[2] * w[2] + w[0] * e1[0];
  const double det = a * c - b * b, det2 = det * det, det3 = det2 * det;
  const double inv = 1. / det;
  const double s = (b * e - c * d) * inv, t = (b * d - a * e) * inv;
  const double u = 1 - (s + t);
  double q[3], dist2 = 0;
  for (int k = 0; k < 3; k++) {
    q[k] = -P[k] + V1[k] * s + V2[k] * t + V0[k] * u;
    dist2 += q[k] * q[k];
  }

  const selector E0 = {2, 1}, E1 = {3, 1}, W = {1, 0};
  double ag[12], bg[12], cg[12], dg[12], eg[12];
  double aH[4][4], bH[4][4], cH[4][4], dH[4][4], eH[4][4];
  bilinear(E0, E0, e0, e0, ag, aH);
  bilinear(E0, E1, e0, e1, bg, bH);
  bilinear(E1, E1, e1, e1, cg, cH);
  bilinear(E0, W, e0, w, dg, dH);
  bilinear(E1, W, e1, w, eg, eH);

  double s1[12], t1[12], u1[12], det1[12];
  for (int i = 0; i < 12; i++) {
    det1[i] = c * ag[i] + a * cg[i] - 2 * b * bg[i];
    s1[i] = ((c * d - b * e) * det1[i]) / det2 + ((e * bg[i] + b * eg[i]) - (d * cg[i] + c * dg[i])) / det;
    t1[i] = ((a * e - b * d) * det1[i]) / det2 + ((d * bg[i] + b * dg[i]) - (a * eg[i] + e * ag[i])) / det;
    u1[i] = -(s1[i] + t1[i]);
  }
  /* dq_k/dx_i */
  double J[3][12];
  for (int k = 0; k < 3; k++)
    for (int i = 0; i < 12; i++) {
      double v = V1[k] * s1[i] + V2[k] * t1[i] + V0[k] * u1[i];
      if (i == k) v -= 1;
      if (i == 3 + k) v += u;
      if (i == 6 + k) v += s;
      if (i == 9 + k) v += t;
      J[k][i] = v;
    }
  for (int i = 0; i < 12; i++) fd[i] = 2 * (q[0] * J[0][i] + q[1] * J[1][i] + q[2] * J[2][i]);

  for (int i = 0; i < 12; i++)
    for (int j = 0; j < 12; j++) {
      const int same = (i % 3) == (j % 3);
      const int bi = i / 3, bj = j / 3;
      const double a2 = same ? aH[bi][bj] : 0, b2 = same ? bH[bi][bj] : 0;
      const double c2 = same ? cH[bi][bj] : 0, d2 = same ? dH[bi][bj] : 0;
      const double e2 = same ? eH[bi][bj] : 0;
      const double det2ij = -2 * bg[i] * bg[j] + ag[j] * cg[i] + ag[i] * cg[j] + c * a2 - 2 * b * b2 + a * c2;
      const double sN = -(c * d) + b * e, tN = b * d - a * e;
      const double s2 =
          (-(cg[j] * dg[i]) - cg[i] * dg[j] + bg[j] * eg[i] + bg[i] * eg[j] + e * b2 - d * c2 - c * d2 + b * e2) / det -
          ((det1[j] * (e * bg[i] - d * cg[i] - c * dg[i] + b * eg[i])) +
           (det1[i] * (e * bg[j] - d * cg[j] - c * dg[j] + b * eg[j])) + (sN * det2ij)) / det2 +
          (2 * sN * det1[i] * det1[j]) / det3;
      const double t2 =
          (bg[j] * dg[i] + bg[i] * dg[j] - ag[j] * eg[i] - ag[i] * eg[j] - e * a2 + d * b2 + b * d2 - a * e2) / det -
          ((det1[j] * (-(e * ag[i]) + d * bg[i] + b * dg[i] - a * eg[i])) +
           (det1[i] * (-(e * ag[j]) + d * bg[j] + b * dg[j] - a * eg[j])) + (tN * det2ij)) / det2 +
          (2 * tN * det1[i] * det1[j]) / det3;
      const double u2 = -(s2 + t2);
      double acc = 0;
      for (int k = 0; k < 3; k++) {
        double q2 = V1[k] * s2 + V2[k] * t2 + V0[k] * u2;
        if (i == 3 + k) q2 += u1[j];
        if (j == 3 + k) q2 += u1[i];
        if (i == 6 + k) q2 += s1[j];
        if (j == 6 + k) q2 += s1[i];
        if (i == 9 + k) q2 += t1[j];
        if (j == 9 + k) q2 += t1[i];
        acc += J[k][i] * J[k][j] + q[k] * q2;
      }
      sd[i * 12 + j] = 2 * acc;
    }
  return dist2;
}

/* pt, point_triange_v2.h:589-841: Voronoi-region selection of the closest
 * feature (Eberly's regions 0-6) and the matching distance function.
 * branch: 0 interior, 1 vertex v1, 2 vertex v2, 3 vertex v0, 4 edge v0-v2,
 * 5 edge v0-v1, 6/7 edge v1-v2. */
double orc_pt(const double x[12], double fd[12], double sd[144], double *s_out,
              double *t_out, int *branch) {
  memset(fd, 0, 12 * sizeof(double));
  memset(sd, 0, 144 * sizeof(double));
  const double *P = x, *V0 = x + 3, *V1 = x + 6, *V2 = x + 9;
  double e0[3], e1[3], w[3];
  for (int k = 0; k < 3; k++) {
    e0[k] = -V0[k] + V1[k];
    e1[k] = -V0[k] + V2[k];
    w[k] = -P[k] + V0[k];
  }
  /* b, c and e are summed over y, z, x and a, d over x, y, z, the order in
   * which point_triange_v2.h:605-610 writes them */
  const double a = e0[0] * e0[0] + e0[1] * e0[1] + e0[2] * e0[2];
  const double b = e1[1] * e0[1] + e1[2] * e0[2] + e0[0] * e1[0];
  const double c = e1[1] * e1[1] + e1[2] * e1[2] + e1[0] * e1[0];
  const double d = w[0] * e0[0] + w[1] * e0[1] + w[2] * e0[2];
  const double e = e1[1] * w[1] + e1[2] * w[2] + w[0] * e1[0];
  const double det = a * c - b * b;
  double s = b * e - c * d, t = b * d - a * e, r;
  int br = -1;

  if (s + t <= det) {
    if (s < 0) {
      if (t < 0 && d < 0) { /* region 4, toward edge v0-v1 */
        t = 0;
        if (-d >= a) { br = 1; s = 1; r = pt_vv(x, 0, 2, fd, sd); }
        else { br = 5; s = -d / a; r = pt_ve(x, 2, 1, fd, sd); }
      } else { /* region 4 with d >= 0, or region 3: edge v0-v2 */
        s = 0;
        if (e >= 0) { br = 3; t = 0; r = pt_vv(x, 0, 1, fd, sd); }
        else if (-e >= c) { br = 2; t = 1; r = pt_vv(x, 0, 3, fd, sd); }
        else { br = 4; t = -e / c; r = pt_ve(x, 3, 1, fd, sd); }
      }
    } else if (t < 0) { /* region 5 */
      t = 0;
      if (d >= 0) { br = 3; s = 0; r = pt_vv(x, 0, 1, fd, sd); }
      else if (-d >= a) { br = 1; s = 1; r = pt_vv(x, 0, 2, fd, sd); }
      else { br = 5; s = -d / a; r = pt_ve(x, 1, 2, fd, sd); }
    } else { /* region 0 */
      br = 0;
      const double inv = (1) / det;
      s *= inv;
      t *= inv;
      r = pt_plane(x, fd, sd);
    }
  } else {
    if (s < 0) { /* region 2 */
      const double t0 = b + d, t1 = c + e;
      if (t1 > t0) {
        const double num = t1 - t0, den = a - 2 * b + c;
        if (num >= den) { br = 1; s = 1; t = 0; r = pt_vv(x, 0, 2, fd, sd); }
        else { br = 6; s = num / den; t = 1 - s; r = pt_ve(x, 2, 3, fd, sd); }
      } else {
        s = 0;
        if (t1 <= 0) { br = 2; t = 1; r = pt_vv(x, 0, 3, fd, sd); }
        else if (e >= 0) { br = 3; t = 0; r = pt_vv(x, 0, 1, fd, sd); }
        else { br = 4; t = -e / c; r = pt_ve(x, 1, 3, fd, sd); }
      }
    } else if (t < 0) { /* region 6 */
      const double t0 = b + e, t1 = a + d;
      if (t1 > t0) {
        const double num = t1 - t0, den = a - 2 * b + c;
        if (num >= den) { br = 2; t = 1; s = 0; r = pt_vv(x, 0, 3, fd, sd); }
        else { br = 7; t = num / den; s = 1 - t; r = pt_ve(x, 2, 3, fd, sd); }
      } else {
        t = 0;
        if (t1 <= 0) { br = 1; s = 1; r = pt_vv(x, 0, 2, fd, sd); }
        else if (d >= 0) { br = 3; s = 0; r = pt_vv(x, 0, 1, fd, sd); }
        else { br = 5; s = -d / a; r = pt_ve(x, 1, 2, fd, sd); }
      }
    } else { /* region 1 */
      const double num = c + e - b - d;
      if (num <= 0) { br = 2; s = 0; t = 1; r = pt_vv(x, 0, 3, fd, sd); }
      else {
        const double den = a - 2 * b + c;
        if (num >= den) { br = 1; s = 1; t = 0; r = pt_vv(x, 0, 2, fd, sd); }
        else { br = 6; s = num / den; t = 1 - s; r = pt_ve(x, 2, 3, fd, sd); }
      }
    }
  }
  *s_out = s;
  *t_out = t;
  *branch = br;
  return r;
}

/* dtn, collision_kernels9/dist_node2tri.h:14-129 (clamped barycentric
 * closest point; the region-6 sub-case keeps the reference's clamp of -e/c). */
static double clamp01(double n) { return n <= 0 ? 0 : n >= 1 ? 1 : n; }
double orc_dtn(const double f[9], const double p[3]) {
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
      if (t1 > t0) {
        s = clamp01((t1 - t0) / (a - 2 * b + c));
        t = 1 - s;
      } else {
        t = clamp01(-e / c);
        s = 0;
      }
    } else if (t < 0) {
      if (a + d > b + e) {
        s = clamp01((c + e - b - d) / (a - 2 * b + c));
        t = 1 - s;
      } else {
        s = clamp01(-e / c);
        t = 0;
      }
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

/* ------------------------------------------------------------------------ */
/* Narrow phase, collision_kernels9/narrowphase.h:3-155                       */
/* ------------------------------------------------------------------------ */

/* inverse of [x1-x0, x2-x0, x3-x0] (Bvalues, :3-33) */
static void tet_inverse(const double *x, double b[9]) {
  const double a11 = x[3] - x[0], a12 = x[6] - x[0], a13 = x[9] - x[0];
  const double a21 = x[4] - x[1], a22 = x[7] - x[1], a23 = x[10] - x[1];
  const double a31 = x[5] - x[2], a32 = x[8] - x[2], a33 = x[11] - x[2];
  const double det = a31 * (-a13 * a22 + a12 * a23) + a32 * (a13 * a21 - a11 * a23) +
                     a33 * (-a12 * a21 + a11 * a22);
  b[0] = (-a23 * a32 + a22 * a33) / det;
  b[1] = (a13 * a32 - a12 * a33) / det;
  b[2] = (-a13 * a22 + a12 * a23) / det;
  b[3] = (a23 * a31 - a21 * a33) / det;
  b[4] = (-a13 * a31 + a11 * a33) / det;
  b[5] = (a13 * a21 - a11 * a23) / det;
  b[6] = (-a22 * a31 + a21 * a32) / det;
  b[7] = (a12 * a31 - a11 * a32) / det;
  b[8] = (-a12 * a21 + a11 * a22) / det;
}
/* strict barycentric inclusion with margin 1e-10 (ctest, :35-44) */
static int tet_contains(const double b[9], double x, double y, double z) {
  const double eps = 1E-10;
  const double y1 = x * b[0] + y * b[1] + z * b[2];
  const double y2 = x * b[3] + y * b[4] + z * b[5];
  const double y3 = x * b[6] + y * b[7] + z * b[8];
  return (y1 > eps && y2 > eps && y3 > eps && (y1 + y2 + y3) < (1 - eps));
}

int orc_narrow_mask(const double xa[12], const double xb[12], const int na[4],
                    const int nb[4]) {
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      if (na[i] == nb[j]) return 0;
  double ba[9], bb[9];
  tet_inverse(xa, ba);
  tet_inverse(xb, bb);
  int m = 0;
  for (int k = 0; k < 4; k++)
    if (tet_contains(ba, xb[3 * k] - xa[0], xb[3 * k + 1] - xa[1], xb[3 * k + 2] - xa[2]))
      m |= 1 << k;
  for (int k = 0; k < 4; k++)
    if (tet_contains(bb, xa[3 * k] - xb[0], xa[3 * k + 1] - xb[1], xa[3 * k + 2] - xb[2]))
      m |= 16 << k;
  return m;
}

void orc_narrow_phase(int n_pairs, const int *pairs, const int *selem,
                      const double *xt, int *masks) {
  for (int i = 0; i < n_pairs; i++) {
    double xa[12], xb[12];
    const int *na = selem + 4 * pairs[2 * i], *nb = selem + 4 * pairs[2 * i + 1];
    for (int k = 0; k < 4; k++)
      for (int c = 0; c < 3; c++) {
        xa[3 * k + c] = xt[3 * na[k] + c];
        xb[3 * k + c] = xt[3 * nb[k] + c];
      }
    masks[i] = orc_narrow_mask(xa, xb, na, nb);
  }
}

/* kDOP24.Expand(x, y, z) (kDOP24.cs:115-141): the 12 slab directions in the
 * reference's order, lower bounds d0..d11, upper bounds d12..d23. */
static void kdop_expand(double d[24], double x, double y, double z) {
  const double pr[12] = {x, y, z, x + y, x + z, y + z, x - y, x - z, y - z, x + y - z, x + z - y, y + z - x};
  for (int k = 0; k < 12; k++) {
    if (pr[k] < d[k]) d[k] = pr[k];
    if (pr[k] > d[12 + k]) d[12 + k] = pr[k];
  }
}

/* kDOP24.Overlaps (kDOP24.cs:84-113). */
static int kdop_overlaps(const double *a, const double *b) {
  for (int k = 0; k < 12; k++)
    if (a[k] > b[12 + k] || a[12 + k] < b[k]) return 0;
  return 1;
}

int orc_kdop_pairs(int n_selem, const int *selem, const double *xt, int *out, long long cap) {
  double *d = (double *)malloc(sizeof(double) * 24 * (size_t)(n_selem > 0 ? n_selem : 1));
  if (!d) return -1;
  for (int e = 0; e < n_selem; e++) {
    double *q = d + 24 * (size_t)e;
    for (int k = 0; k < 12; k++) {  /* Reset(): +max / -max (kDOP24.cs:60-64) */
      q[k] = DBL_MAX;
      q[12 + k] = -DBL_MAX;
    }
    for (int v = 0; v < 4; v++) {
      const int n = selem[4 * e + v];
      kdop_expand(q, xt[3 * n], xt[3 * n + 1], xt[3 * n + 2]);
    }
  }
  long long np = 0;
  for (int a = 0; a < n_selem; a++)
    for (int b = a + 1; b < n_selem; b++)
      if (kdop_overlaps(d + 24 * (size_t)a, d + 24 * (size_t)b)) {
        if (np >= cap) {
          free(d);
          return -1;
        }
        out[2 * np] = a;
        out[2 * np + 1] = b;
        np++;
      }
  free(d);
  return (int)np;
}

typedef struct {
  unsigned long long key;
  int elem;
} cell_entry;
static int cmp_entry(const void *a, const void *b) {
  const cell_entry *x = (const cell_entry *)a, *y = (const cell_entry *)b;
  if (x->key != y->key) return (x->key > y->key) - (x->key < y->key);
  return (x->elem > y->elem) - (x->elem < y->elem);
}
static int cmp_ull(const void *a, const void *b) {
  const unsigned long long x = *(const unsigned long long *)a, y = *(const unsigned long long *)b;
  return (x > y) - (x < y);
}

static int vert_in_box(const int *n, const double *xt, const double *lo, const double *hi) {
  for (int v = 0; v < 4; v++) {
    const double *p = xt + 3 * n[v];
    if (p[0] >= lo[0] && p[0] <= hi[0] && p[1] >= lo[1] && p[1] <= hi[1] && p[2] >= lo[2] && p[2] <= hi[2])
      return 1;
  }
  return 0;
}

long long orc_candidate_pairs(int n, const int *selem, const int *group, const double *xt, double pad,
                              int *out, long long cap) {
  if (n < 2) return 0;
  double *lo = (double *)malloc(sizeof(double) * 6 * (size_t)n), *hi = lo + 3 * (size_t)n;
  cell_entry *ent = (cell_entry *)malloc(sizeof(cell_entry) * 8 * (size_t)n);
  if (!lo || !ent) {
    free(lo);
    free(ent);
    return -1;
  }
  double cell = 0.0, base[3] = {DBL_MAX, DBL_MAX, DBL_MAX};
  for (int e = 0; e < n; e++)
    for (int k = 0; k < 3; k++) {
      double a = DBL_MAX, b = -DBL_MAX;
      for (int v = 0; v < 4; v++) {
        const double x = xt[3 * selem[4 * e + v] + k];
        a = x < a ? x : a;
        b = x > b ? x : b;
      }
      lo[3 * e + k] = a - pad;
      hi[3 * e + k] = b + pad;
      if (hi[3 * e + k] - lo[3 * e + k] > cell) cell = hi[3 * e + k] - lo[3 * e + k];
      if (lo[3 * e + k] < base[k]) base[k] = lo[3 * e + k];
    }
  if (!(cell > 0)) cell = 1.0;
  long long m = 0;
  for (int e = 0; e < n; e++) {
    long long c0[3], c1[3];
    for (int k = 0; k < 3; k++) {
      c0[k] = (long long)floor((lo[3 * e + k] - base[k]) / cell);
      c1[k] = (long long)floor((hi[3 * e + k] - base[k]) / cell);
    }
    for (long long x = c0[0]; x <= c1[0] && x <= c0[0] + 1; x++)
      for (long long y = c0[1]; y <= c1[1] && y <= c0[1] + 1; y++)
        for (long long z = c0[2]; z <= c1[2] && z <= c0[2] + 1; z++) {
          ent[m].key = ((unsigned long long)x << 42) | ((unsigned long long)y << 21) | (unsigned long long)z;
          ent[m].elem = e;
          m++;
        }
  }
  qsort(ent, (size_t)m, sizeof(cell_entry), cmp_entry);
  long long np = 0, pcap = 16 * (long long)n + 1024;
  unsigned long long *pk = (unsigned long long *)malloc(sizeof(unsigned long long) * (size_t)pcap);
  for (long long i = 0; i < m && pk; i++)
    for (long long j = i + 1; j < m && ent[j].key == ent[i].key; j++) {
      int a = ent[i].elem, b = ent[j].elem;
      if (a > b) {
        const int t = a;
        a = b;
        b = t;
      }
      if (group && group[a] == group[b]) continue;
      int ov = 1;
      for (int k = 0; k < 3; k++)
        if (!(lo[3 * a + k] <= hi[3 * b + k] && lo[3 * b + k] <= hi[3 * a + k])) ov = 0;
      if (!ov) continue;
      const int *na = selem + 4 * a, *nb = selem + 4 * b;
      int shared = 0;
      for (int p = 0; p < 4; p++)
        for (int q = 0; q < 4; q++) shared |= na[p] == nb[q];
      if (shared) continue;
      if (!vert_in_box(na, xt, lo + 3 * b, hi + 3 * b) && !vert_in_box(nb, xt, lo + 3 * a, hi + 3 * a)) continue;
      if (np == pcap) {
        pcap *= 2;
        unsigned long long *q = (unsigned long long *)realloc(pk, sizeof(unsigned long long) * (size_t)pcap);
        if (!q) {
          free(pk);
          pk = NULL;
          break;
        }
        pk = q;
      }
      pk[np++] = ((unsigned long long)(unsigned)a << 32) | (unsigned)b;
    }
  free(lo);
  free(ent);
  if (!pk) return -1;
  qsort(pk, (size_t)np, sizeof(unsigned long long), cmp_ull);
  long long u = 0;
  for (long long i = 0; i < np; i++) {
    if (i > 0 && pk[i] == pk[i - 1]) continue;
    if (u >= cap) {
      free(pk);
      return -1;
    }
    out[2 * u] = (int)(pk[i] >> 32);
    out[2 * u + 1] = (int)(pk[i] & 0xffffffffu);
    u++;
  }
  free(pk);
  return u;
}

static int cmp_ll(const void *a, const void *b) {
  const long long x = *(const long long *)a, y = *(const long long *)b;
  return (x > y) - (x < y);
}

/* Set expansion of GPU_Functionality.cs:566-580 (canonical ascending order of
 * (node, element) instead of hash insertion order) followed by
 * kFindClosestFace, narrowphase.h:159-201 (strict minimum: the first face in
 * adjacency order wins ties). */
int orc_impacts(int n_pairs, const int *pairs, const int *masks,
                const int *selem, const int *adj_off, const int *adj_faces,
                const int *faces, const double *xt, int *out, int cap) {
  long long *keys = (long long *)malloc(sizeof(long long) * (size_t)(8 * (n_pairs > 0 ? n_pairs : 1)));
  int n = 0;
  for (int i = 0; i < n_pairs; i++) {
    const int m = masks[i];
    if (!m) continue;
    const int ea = pairs[2 * i], eb = pairs[2 * i + 1];
    for (int k = 0; k < 4; k++)
      if (m & (1 << k)) keys[n++] = ((long long)selem[4 * eb + k] << 32) | (unsigned)ea;
    for (int k = 0; k < 4; k++)
      if (m & (16 << k)) keys[n++] = ((long long)selem[4 * ea + k] << 32) | (unsigned)eb;
  }
  qsort(keys, (size_t)n, sizeof(long long), cmp_ll);
  int u = 0;
  for (int i = 0; i < n; i++)
    if (i == 0 || keys[i] != keys[i - 1]) keys[u++] = keys[i];
  if (u > cap) {
    free(keys);
    return -1;
  }
  for (int i = 0; i < u; i++) {
    const int node = (int)(keys[i] >> 32), el = (int)(keys[i] & 0xffffffffLL);
    const double *p = xt + 3 * node;
    int best = -1;
    double bestd = 0;
    for (int q = adj_off[el]; q < adj_off[el + 1]; q++) {
      const int fc = adj_faces[q];
      double fx[9];
      for (int v = 0; v < 3; v++)
        for (int c = 0; c < 3; c++) fx[3 * v + c] = xt[3 * faces[3 * fc + v] + c];
      const double dd = orc_dtn(fx, p);
      if (q == adj_off[el] || dd < bestd) {
        best = fc;
        bestd = dd;
      }
    }
    out[4 * i] = node;
    out[4 * i + 1] = faces[3 * best];
    out[4 * i + 2] = faces[3 * best + 1];
    out[4 * i + 3] = faces[3 * best + 2];
  }
  free(keys);
  return u;
}

/* kCollisionResponseForce body, collision_response.h:54-114:
 * F = k/2 grad_p(d^2); fi = (-F, w0 F, w1 F, w2 F); H = k/2 Hess(d^2). */
int orc_contact_local(const orc_prms *p, const double x[12], double lhs[144],
                      double rhs[12]) {
  double fd[12], sd[144], s, t;
  int br;
  const double dsq = orc_pt(x, fd, sd, &s, &t, &br);
  const double w[3] = {1 - (s + t), s, t};
  if (!(dsq > p->DistanceEpsilon * p->DistanceEpsilon)) return 0;
  const double F[3] = {p->penaltyK * 0.5 * fd[0], p->penaltyK * 0.5 * fd[1],
                       p->penaltyK * 0.5 * fd[2]};
  for (int k = 0; k < 3; k++) {
    rhs[k] = -F[k];
    for (int v = 0; v < 3; v++) rhs[3 + 3 * v + k] = w[v] * F[k];
  }
  for (int i = 0; i < 12; i++)
    for (int j = i; j < 12; j++)
      lhs[i * 12 + j] = lhs[j * 12 + i] = p->penaltyK * sd[i * 12 + j] / 2;
  return 1;
}

/* ------------------------------------------------------------------------ */
/* Sparsity pattern, v3Library/Simulation/LinearSystem/CSRDictionary.cs      */
/* ------------------------------------------------------------------------ */

/* Static pairs (MeshCollection.cs:91-109, j >= i) and dynamic pairs
 * (ImplicitModel3.cs:177-196, j > i), union per row, columns ascending
 * (CSRDictionary.cs:64-97).  N = 1 + the largest static row. */
int orc_build_structure(int n_nodes, const int *alt, int n_elem,
                        const int *elem, int n_cz, const int *cz, int n_imp,
                        const int *imp, int *csr_rows, int *csr_cols,
                        int *nnz, long long cap_cols) {
  (void)n_nodes;
  const size_t nk = (size_t)n_elem * 16 + (size_t)n_cz * 36 + (size_t)n_imp * 16 + 1;
  long long *keys = (long long *)malloc(sizeof(long long) * nk);
  size_t n = 0;
  int maxrow = -1;
  for (int u = 0; u < n_elem; u++)
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 4; j++) {
        const int ai = alt[elem[4 * u + i]], aj = alt[elem[4 * u + j]];
        if (ai >= 0 && aj >= 0 && aj >= ai) {
          keys[n++] = ((long long)ai << 32) | (unsigned)aj;
          if (ai > maxrow) maxrow = ai;
        }
      }
  for (int u = 0; u < n_cz; u++)
    for (int i = 0; i < 6; i++)
      for (int j = 0; j < 6; j++) {
        const int ai = alt[cz[6 * u + i]], aj = alt[cz[6 * u + j]];
        if (ai >= 0 && aj >= 0 && aj >= ai) {
          keys[n++] = ((long long)ai << 32) | (unsigned)aj;
          if (ai > maxrow) maxrow = ai;
        }
      }
  for (int u = 0; u < n_imp; u++)
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 4; j++) {
        const int ai = alt[imp[4 * u + i]], aj = alt[imp[4 * u + j]];
        if (ai >= 0 && aj >= 0 && aj > ai) {
          if (ai > maxrow) { free(keys); return -2; } /* row outside the pattern */
          keys[n++] = ((long long)ai << 32) | (unsigned)aj;
        }
      }
  qsort(keys, n, sizeof(long long), cmp_ll);
  size_t u = 0;
  for (size_t i = 0; i < n; i++)
    if (i == 0 || keys[i] != keys[i - 1]) keys[u++] = keys[i];
  const int N = maxrow + 1;
  if (csr_cols && (long long)u > cap_cols) {
    free(keys);
    return -1;
  }
  size_t q = 0;
  for (int r = 0; r < N; r++) {
    csr_rows[r] = (int)q;
    while (q < u && (int)(keys[q] >> 32) == r) {
      if (csr_cols) csr_cols[q] = (int)(keys[q] & 0xffffffffLL);
      q++;
    }
  }
  csr_rows[N] = (int)q;
  *nnz = (int)u;
  free(keys);
  return N;
}

/* CSRDictionary indexer (CSRDictionary.cs:99-105), -1 where absent. */
int orc_slot(const int *csr_rows, const int *csr_cols, int N, int i, int j) {
  if (i < 0 || i >= N) return -1;
  int lo = csr_rows[i], hi = csr_rows[i + 1] - 1;
  while (lo <= hi) {
    const int m = (lo + hi) / 2;
    if (csr_cols[m] == j) return m;
    if (csr_cols[m] < j) lo = m + 1;
    else hi = m - 1;
  }
  return -1;
}

/* TransferPCSR / collisionResponse index maps, GPU_Functionality.cs:355-368,
 * :388-401 and :647-662. */
void orc_pcsr(int n_units, int k, const int *unit_nodes, const int *alt,
              const int *csr_rows, const int *csr_cols, int N, int *out) {
  const int w = k * k + k;
  for (int u = 0; u < n_units; u++) {
    const int *nd = unit_nodes + (size_t)u * k;
    int *o = out + (size_t)u * w;
    for (int i = 0; i < k; i++) {
      const int ai = alt[nd[i]];
      for (int j = 0; j < k; j++) {
        const int aj = alt[nd[j]];
        o[i * k + j] = (ai >= 0 && aj >= 0 && aj >= ai) ? orc_slot(csr_rows, csr_cols, N, ai, aj) : -1;
      }
      o[k * k + i] = ai >= 0 ? ai : -1;
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Assembly (the scatter of AssembleBCSR12/18, element_kernels2.h:162-189,   */
/* cz_kernels.h:177-203, collision_response.h:6-33)                          */
/* ------------------------------------------------------------------------ */

static void scatter(int k, const int *pcsr, const double *lhs, const double *r,
                    double *vals, double *rhs) {
  const int n = 3 * k;
  for (int i = 0; i < k; i++) {
    for (int j = 0; j < k; j++) {
      const int slot = pcsr[i * k + j];
      if (slot < 0) continue;
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
          vals[(size_t)slot * 9 + 3 * a + b] += lhs[(3 * i + a) * n + 3 * j + b];
    }
    const int row = pcsr[k * k + i];
    if (row >= 0)
      for (int a = 0; a < 3; a++) rhs[(size_t)row * 3 + a] += r[3 * i + a];
  }
}

void orc_assemble(const orc_prms *p, double h, int n_nodes, const double *x0,
                  const double *un, const double *vn, const double *an,
                  const double *xt, int n_elem, const int *elem,
                  const int *elem_pcsr, int n_cz, const int *cz,
                  const int *cz_pcsr, const orc_ppr *cz_ppr,
                  const double *pmax, const double *tmax, int n_imp,
                  const int *imp, const int *imp_pcsr, double *vals,
                  double *rhs, double *nodeF, double *tent, int *flags,
                  double *avg) {
  (void)n_nodes;
  for (int u = 0; u < n_elem; u++) {
    double lx0[12], lun[12], lvn[12], lan[12], lhs[144], r[12];
    for (int i = 0; i < 4; i++)
      for (int c = 0; c < 3; c++) {
        const int nd = elem[4 * u + i];
        lx0[3 * i + c] = x0[3 * nd + c];
        lun[3 * i + c] = un[3 * nd + c];
        lvn[3 * i + c] = vn[3 * nd + c];
        lan[3 * i + c] = an[3 * nd + c];
      }
    orc_elem_local(p, h, lx0, lun, lvn, lan, lhs, r);
    for (int i = 0; i < 4; i++)
      for (int c = 0; c < 3; c++) nodeF[3 * elem[4 * u + i] + c] += r[3 * i + c];
    scatter(4, elem_pcsr + (size_t)u * 20, lhs, r, vals, rhs);
  }
  for (int u = 0; u < n_cz; u++) {
    double lx0[18], lun[18], keff[324], r[18];
    for (int i = 0; i < 6; i++)
      for (int c = 0; c < 3; c++) {
        const int nd = cz[6 * u + i];
        lx0[3 * i + c] = x0[3 * nd + c];
        lun[3 * i + c] = un[3 * nd + c];
      }
    const orc_ppr *q = cz_ppr ? cz_ppr + u : &p->ppr;
    orc_cz_local(p, q, lx0, lun, pmax + 3 * u, tmax + 3 * u, keff, r, tent + 2 * u,
                 flags + 3 * u, avg + 4 * u);
    if (flags[3 * u + 2]) continue; /* failed: nothing scattered (:424) */
    scatter(6, cz_pcsr + (size_t)u * 42, keff, r, vals, rhs);
  }
  for (int u = 0; u < n_imp; u++) {
    const int *pc = imp_pcsr + (size_t)u * 20;
    if (pc[16] < 0 && pc[17] < 0 && pc[18] < 0 && pc[19] < 0) continue; /* :47-51 */
    double x[12], lhs[144], r[12];
    for (int i = 0; i < 4; i++)
      for (int c = 0; c < 3; c++) x[3 * i + c] = xt[3 * imp[4 * u + i] + c];
    if (!orc_contact_local(p, x, lhs, r)) continue;
    for (int i = 0; i < 4; i++)
      for (int c = 0; c < 3; c++) nodeF[3 * imp[4 * u + i] + c] += r[3 * i + c];
    scatter(4, pc, lhs, r, vals, rhs);
  }
}

/* ------------------------------------------------------------------------ */
/* Newmark kinematics, v3Library/Geometry/Node.cs                             */
/* ------------------------------------------------------------------------ */

void orc_newmark_infer(int n, double h, double beta, double gamma,
                       const double *x0, const double *u, const double *v,
                       const double *a, const double *du, double *un,
                       double *vn, double *an, double *xt) {
  for (int i = 0; i < 3 * n; i++) {
    un[i] = u[i] + du[i];
    an[i] = a[i] * (1.0 - 1.0 / (2 * beta)) + du[i] / (h * h * beta) + v[i] * (-1.0 / (h * beta));
    vn[i] = v[i] + h * ((1.0 - gamma) * a[i] + gamma * an[i]);
    xt[i] = x0[i] + un[i];
  }
}

void orc_newmark_accept(int n, double h, const double *x0, double *u,
                        double *v, double *a, const double *un, double *du,
                        double *xc) {
  for (int i = 0; i < 3 * n; i++) {
    const double vnew = (un[i] - u[i]) / h;
    a[i] = (vnew - v[i]) / h;
    v[i] = vnew;
    u[i] = un[i];
    xc[i] = x0[i] + u[i];
    du[i] = 0;
  }
}
