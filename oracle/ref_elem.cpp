/* Host build of the reference element module (elem_kernels9/kernel.cu and the
 * headers it includes), read in place from the reference checkout through
 * ref_shim/shim.h. TEST INFRASTRUCTURE ONLY (oracle/_ref): a checker and the
 * timed "reference" CPU baseline, never part of the product path.
 *
 * Entry points:
 *   ref_elem_set_constants  -> the __constant__ block of elem_constants.h:2-5
 *                              (set by GPU_Functionality.cs:157-165)
 *   ref_elem_F_and_Df       -> F_and_Df_Corotational, element_kernels2.h:19-159
 *   ref_elem_kernel         -> kelElementElasticityForce, element_kernels2.h:195-263,
 *                              one OpenMP iteration per unit (launch shape of
 *                              GPU_Functionality.cs:448-454)
 */
#include "shim.h"
#include <omp.h>

namespace icf_ref_elem {
#include "kernel.cu"
}

namespace {
struct ElemConsts {
  double E[6][6], M[12][12];
  double beta, gamma, dm, ds, rho, g, Y;
};
ElemConsts g_c;

void load_thread_constants() {
  using namespace icf_ref_elem;
  std::memcpy(E, g_c.E, sizeof(E));
  std::memcpy(M, g_c.M, sizeof(M));
  NewmarkBeta = g_c.beta;
  NewmarkGamma = g_c.gamma;
  dampingMass = g_c.dm;
  dampingStiffness = g_c.ds;
  rho = g_c.rho;
  gravity = g_c.g;
  YoungsModulus = g_c.Y;
}
}  // namespace

extern "C" {

void ref_elem_set_constants(const double *E36, const double *M144, double beta,
                            double gamma, double dm, double ds, double rho,
                            double g, double Y) {
  std::memcpy(g_c.E, E36, sizeof(g_c.E));
  std::memcpy(g_c.M, M144, sizeof(g_c.M));
  g_c.beta = beta;
  g_c.gamma = gamma;
  g_c.dm = dm;
  g_c.ds = ds;
  g_c.rho = rho;
  g_c.g = g;
  g_c.Y = Y;
}

/* Unscattered per-unit result: f[12], Df[144] (row-major), V. */
void ref_elem_F_and_Df(int n, const double *x0, const double *un, double *f,
                       double *Df, double *V) {
#pragma omp parallel
  {
    load_thread_constants();
#pragma omp for schedule(static)
    for (int e = 0; e < n; e++) {
      double lx0[12], lun[12], lf[12] = {}, lDf[12][12] = {}, lV = 0;
      for (int i = 0; i < 12; i++) {
        lx0[i] = x0[12 * e + i];
        lun[i] = un[12 * e + i];
      }
      icf_ref_elem::F_and_Df_Corotational(lx0, lun, lf, lDf, lV);
      for (int i = 0; i < 12; i++) f[12 * e + i] = lf[i];
      std::memcpy(Df + 144 * e, lDf, sizeof(lDf));
      V[e] = lV;
    }
  }
}

/* Whole kernel over all units with the reference's strided layouts. */
void ref_elem_kernel(const int *ie, double *dn, double h, double *vals,
                     double *rhs, int nElems, int el_stride, int nd_stride,
                     int nthreads) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
  {
    load_thread_constants();
#pragma omp for schedule(static)
    for (int e = 0; e < nElems; e++) {
      icf_shim_set_thread(e);
      icf_ref_elem::kelElementElasticityForce(ie, dn, h, vals, rhs, nElems,
                                              el_stride, nd_stride);
    }
  }
}

}  // extern "C"
