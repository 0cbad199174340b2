/* Host build of the reference cohesive-zone module (cz_kernels9/kernel.cu and
 * the headers it includes), read in place through ref_shim/shim.h.
 * TEST INFRASTRUCTURE ONLY (oracle/_ref).
 *
 * Entry points:
 *   ref_cz_set_constants -> __constant__ block of cz_constants.h:2-17
 *                           (set by GPU_Functionality.cs:169-193)
 *   ref_cz_ppr           -> Tn_, Tt_, Dnn_, Dtt_, Dnt_ (PPR_math.h:2-57)
 *   ref_cz_law           -> cohesive_law_thermodynamically_consistent
 *                           (cz_kernels.h:37-174)
 *   ref_cz_kernel        -> kczCZForce (cz_kernels.h:210-434), one OpenMP
 *                           iteration per unit; optional per-CZ strengths
 *                           (f_tn, f_tt, deln, delt) replace the globals for
 *                           that unit, which is how a per-boundary strength
 *                           field is evaluated with the unmodified kernel.
 */
#include "shim.h"
#include <omp.h>

namespace icf_ref_cz {
#include "kernel.cu"
}

namespace {
/* order: NewmarkBeta NewmarkGamma dampingMass dampingStiffness rho gravity
 *        G_fn G_ft f_tn f_tt alpha beta rn rt p_m p_n deln delt pMtn pMnt
 *        gam_n gam_t  (22 scalars), then M[144], B[162], sf[9] */
struct CzConsts {
  double s[22];
  double M[12][12];
  double B[3][3][18];
  double sf[3][3];
};
CzConsts g_c;

void load_thread_constants() {
  using namespace icf_ref_cz;
  const double *s = g_c.s;
  NewmarkBeta = s[0]; NewmarkGamma = s[1]; dampingMass = s[2];
  dampingStiffness = s[3]; rho = s[4]; gravity = s[5];
  G_fn = s[6]; G_ft = s[7]; f_tn = s[8]; f_tt = s[9];
  alpha = s[10]; beta = s[11]; rn = s[12]; rt = s[13];
  p_m = s[14]; p_n = s[15]; deln = s[16]; delt = s[17];
  pMtn = s[18]; pMnt = s[19]; gam_n = s[20]; gam_t = s[21];
  std::memcpy(M, g_c.M, sizeof(M));
  std::memcpy(B, g_c.B, sizeof(B));
  std::memcpy(sf, g_c.sf, sizeof(sf));
}
}  // namespace

extern "C" {

void ref_cz_set_constants(const double *scalars22, const double *M144,
                          const double *B162, const double *sf9) {
  std::memcpy(g_c.s, scalars22, sizeof(g_c.s));
  std::memcpy(g_c.M, M144, sizeof(g_c.M));
  std::memcpy(g_c.B, B162, sizeof(g_c.B));
  std::memcpy(g_c.sf, sf9, sizeof(g_c.sf));
}

/* out[5*i + k] = Tn_, Tt_, Dnn_, Dtt_, Dnt_ evaluated at (dn[i], dt[i]). */
void ref_cz_ppr(int n, const double *dn, const double *dt, double *out) {
  load_thread_constants();
  for (int i = 0; i < n; i++) {
    out[5 * i + 0] = icf_ref_cz::Tn_(dn[i], dt[i]);
    out[5 * i + 1] = icf_ref_cz::Tt_(dn[i], dt[i]);
    out[5 * i + 2] = icf_ref_cz::Dnn_(dn[i], dt[i]);
    out[5 * i + 3] = icf_ref_cz::Dtt_(dn[i], dt[i]);
    out[5 * i + 4] = icf_ref_cz::Dnt_(dn[i], dt[i]);
  }
}

/* pmax/tmax updated in place; out[6*i+k] = Tn Tt Dnn Dtt Dnt Dtn;
 * flags[2*i] = contact, flags[2*i+1] = failed. */
void ref_cz_law(int n, double *pmax, double *tmax, const double *opn,
                const double *opt, double *out, int *flags) {
  load_thread_constants();
  for (int i = 0; i < n; i++) {
    bool contact = false, failed = false;
    double Tn, Tt, Dnn, Dtt, Dnt, Dtn;
    icf_ref_cz::cohesive_law_thermodynamically_consistent(
        contact, failed, pmax[i], tmax[i], opn[i], opt[i], Tn, Tt, Dnn, Dtt,
        Dnt, Dtn);
    out[6 * i + 0] = Tn; out[6 * i + 1] = Tt; out[6 * i + 2] = Dnn;
    out[6 * i + 3] = Dtt; out[6 * i + 4] = Dnt; out[6 * i + 5] = Dtn;
    flags[2 * i] = contact ? 1 : 0;
    flags[2 * i + 1] = failed ? 1 : 0;
  }
}

void ref_cz_kernel(double *dcz, int *icz, double *dnd, double *vals,
                   double *rhs, double h, int nCZs, int cz_stride,
                   int nd_stride, const double *f_tn_arr,
                   const double *f_tt_arr, const double *deln_arr,
                   const double *delt_arr, int nthreads) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
  {
    load_thread_constants();
#pragma omp for schedule(static)
    for (int c = 0; c < nCZs; c++) {
      if (f_tn_arr) {
        icf_ref_cz::f_tn = f_tn_arr[c];
        icf_ref_cz::f_tt = f_tt_arr[c];
        icf_ref_cz::deln = deln_arr[c];
        icf_ref_cz::delt = delt_arr[c];
      }
      icf_shim_set_thread(c);
      icf_ref_cz::kczCZForce(dcz, icz, dnd, vals, rhs, h, nCZs, cz_stride,
                             nd_stride);
    }
  }
}

}  // extern "C"
