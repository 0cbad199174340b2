// icf_ppr.cuh -- Park-Paulino-Roesler cohesive law on the device.
//
// PPR potential derivatives (cz_kernels9/PPR_math.h:2-57) and the
// thermodynamically consistent law with unload/reload and contact branches
// (cz_kernels9/cz_kernels.h:37-174).  The branch structure is the algorithm
// and is kept; the PPR functions are written as products of one factor per
// axis, and each axis is evaluated once per Gauss point.
#pragma once
#include <cuda_runtime.h>

#include "icf_exact.cuh"

// Law outputs for one Gauss point.
struct icf_law {
  double Tn, Tt, Dnn, Dtt, Dnt;
  bool contact, failed;
};

// ---- axis form of the law -------------------------------------------------------
// Every PPR function is a product of one factor per axis (PPR_math.h:2-57):
//   Tn  = (gam_n/deln)        dN(xn)  fT(xt)      Tt  = (gam_t/delt)        dT(xt)  fN(xn)
//   Dnn = (gam_n/deln^2)      ddN(xn) fT(xt)      Dtt = (gam_t/delt^2)      ddT(xt) fN(xn)
//   Dnt = (gam_n gam_t/(deln delt)) dN(xn) dT(xt)
// with, for the normal axis (alpha, p_m; the tangential one uses beta, p_n),
//   fN  = gam_n (1-x)^a (p/a+x)^p + <phi_n - phi_t>
//   dN  = p (1-x)^a (p/a+x)^(p-1) - a (1-x)^(a-1) (p/a+x)^p
//   ddN = (p^2-p)(1-x)^a (p/a+x)^(p-2) + (a^2-a)(1-x)^(a-2)(p/a+x)^p
//         - 2 a p (1-x)^(a-1) (p/a+x)^(p-1).
// The law only ever evaluates an axis at the current opening, at the
// historical maximum, or at zero, so each Gauss point needs at most four axis
// evaluations (the zero ones are constants).  (1-x)^(a-k) and (p/a+x)^(p-k)
// come from one pow each and exact divisions by (1-x) and (p/a+x).
struct icf_axis {
  double f, d, dd;
  // for the decision bounds (icf_law_bound): md = |p o0 s1| + |a o1 s0| and
  // mf = |gam o0 s0| + |mac|, the magnitudes of the terms of d and f, and k,
  // the rounding error of this evaluation of d and f in units of 2^-53 of
  // those magnitudes
  double md, mf, k;
};

__device__ __forceinline__ icf_axis icf_axis_eval(double a, double p, double gam, double mac,
                                                  double x, int a_int = 0) {
  const double o = 1.0 - x, s = (p / a) + x;
  double o0, o1, o2;
  if (a_int >= 2) {  // integer exponent: (1-x)^(a-2) by repeated products
    o2 = 1.0;
    for (int k = 0; k < a_int - 2; k++) o2 *= o;
    o1 = o2 * o;
    o0 = o1 * o;
  } else if (o > 0) {
    const double io = 1.0 / o;
    o0 = pow(o, a);
    o1 = o0 * io;
    o2 = o1 * io;
  } else {
    o0 = pow(o, a);
    o1 = pow(o, a - 1.0);
    o2 = pow(o, a - 2.0);
  }
  // s = p/a + x > 0 wherever the law evaluates an axis (x >= 0), so s^p is
  // 2^(p log2 s): two library calls, cheaper than the general pow
  const double is = 1.0 / s;
  const double E = p * log2(s);
  const double s0 = exp2(E), s1 = s0 * is, s2 = s1 * is;
  icf_axis r;
  r.f = gam * o0 * s0 + mac;
  r.d = (p * o0 * s1) - (a * o1 * s0);
  r.dd = (p * p - p) * o0 * s2 + (a * a - a) * o2 * s0 - 2.0 * a * p * o1 * s1;
  // o^(a-k): a - 2 products or pow (2 ulp) and a division; s^p: log2 (1 ulp),
  // the product with p and exp2 (2 ulp) give 2 ulp + 3 ulp |p log2 s|
  r.md = fabs(p * o0 * s1) + fabs(a * o1 * s0);
  r.mf = fabs(gam * o0 * s0) + fabs(mac);
  r.k = fabs(a) + 24.0 + 3.0 * fabs(E);
  return r;
}

struct icf_law_c {
  double alpha, beta, p_m, p_n, gam_n, gam_t, pMtn, pMnt, rn, rt;
  icf_axis N0, T0;  // axes at zero opening
  // the reference's dN and dT at zero opening, p S1 - a S0 with S_k =
  // pow(p/a, p - k) from the host C library (PPR_math.h:8-9, 20): the exact
  // difference is 0, so this constant is pure rounding and is taken as the
  // reference computes it
  double zN, zT;
  int alpha_int, beta_int;  // alpha, beta when they are integers in [2, 16], else 0
};

// ---- the law's decisions ----------------------------------------------------------
// The reference compares Tt_ and Tn_ (at the current opening) with -1e-9 and,
// past a fifth of the characteristic opening, with 5 % of the strength
// (cz_kernels.h:43-47, 90-95).  The fast values here are the axis products
// cT dT(xt) fN(xn) and cN dN(xn) fT(xt); their distance from the reference's
// values is bounded by the term magnitudes times the rounding counts of both
// evaluations (the reference's: pow within an ulp, three products).  At a
// zero opening the axis difference dT or dN is pure rounding noise (about
// 1e-10 in traction, against the -1e-9 threshold), so there it is replaced
// by the reference's own constant zT or zN and only the other, well
// conditioned factor is approximate.  A comparison that the bound still
// cannot settle is "undecided": the assembly's CZ kernel counts it
// (EXACT = false) and the library then repeats that assembly with the
// EXACT = true kernel, which settles it on icf_ref_Tt/icf_ref_Tn, the
// reference's expressions with pow correctly rounded (icf_exact.cuh).
__device__ __forceinline__ double icf_law_bound(double c, const icf_axis &own, const icf_axis &other) {
  const double u = 1.1102230246251565e-16;  // 2^-53
  return 2.0 * fabs(c) * own.md * other.mf * (own.k + other.k + 18.0) * u;
}
// the decision value at a zero opening of its own axis: (g/del) z f_other
// with the products rounded as the reference rounds them
__device__ __forceinline__ double icf_law_zero(double g, double del, double z, const icf_axis &other, double &e) {
  const double u = 1.1102230246251565e-16;
  const double pr12 = __dmul_rn(__ddiv_rn(g, del), z);
  e = 2.0 * fabs(pr12) * other.mf * (other.k + 8.0) * u;
  return __dmul_rn(pr12, other.f);
}
__device__ __forceinline__ bool icf_near(double v, double e, double thr) { return fabs(v - thr) <= e; }

// Tn_ and Tt_ at (dn, dt) by the reference expressions (icf_exact.cuh).
__device__ __forceinline__ double2 icf_law_exact_T(const icf_law_c &C, double deln, double delt, double dn,
                                                   double dt) {
  const icf_ppr_k K{C.alpha, C.beta, C.p_m, C.p_n, C.gam_n, C.gam_t, C.pMtn, C.pMnt};
  return make_double2(icf_ref_Tn(K, deln, delt, dn, dt), icf_ref_Tt(K, deln, delt, dn, dt));
}

// The axes at the committed history, N(pmax/deln) and T(tmax/delt).  They only
// change when the damage state does, so the assembly reads them from a cache
// (k_cz_hist) instead of evaluating two of its four axes every iteration.
__device__ __forceinline__ void icf_cz_hist_axes(const icf_law_c &C, double deln, double delt, double pmax,
                                                 double tmax, icf_axis &Np, icf_axis &Tm) {
  Np = icf_axis_eval(C.alpha, C.p_m, C.gam_n, C.pMnt, pmax / deln, C.alpha_int);
  Tm = icf_axis_eval(C.beta, C.p_n, C.gam_t, C.pMtn, tmax / delt, C.beta_int);
}

// cohesive_law_thermodynamically_consistent (cz_kernels.h:37-174) on the axis
// factors, given the history axes Np, Tm of the incoming pmax, tmax; pmax and
// tmax are updated in place.  `undecided` is set when a failure comparison
// could not be settled without the reference's rounding (EXACT = false).
template <bool EXACT>
__device__ inline icf_law icf_cz_law_hist(const icf_law_c &C, double f_tn, double f_tt, double deln,
                                          double delt, const icf_axis &Np, const icf_axis &Tm, double &pmax,
                                          double &tmax, double opn, double opt, bool &undecided) {
  icf_law L;
  L.Tn = L.Tt = L.Dnn = L.Dtt = L.Dnt = 0;
  L.contact = false;
  L.failed = false;
  if (opn > deln || opt > delt) {
    L.failed = true;
    return L;
  }
  const double ideln = 1.0 / deln, idelt = 1.0 / delt;
  const double cN = C.gam_n * ideln, cT = C.gam_t * idelt;
  const double cNN = cN * ideln, cTT = cT * idelt;
  const double cNT = cN * cT;
  L.contact = (opn < 0);
  const double eps_neg = -1e-9;
  const double thr_t = f_tt * 0.05, thr_n = f_tn * 0.05;
  const icf_axis To = icf_axis_eval(C.beta, C.p_n, C.gam_t, C.pMtn, opt * idelt, C.beta_int);
  const bool t_past = opt > delt * C.rt / 5;
  if (L.contact) {
    if (pmax != 0) {
      const double peak = cN * Np.d * Tm.f;           // Tn_(pmax, tmax)
      L.Tn = peak * opn / pmax;
      L.Dnn = peak / pmax;
    } else {
      L.Dnn = cNN * C.N0.dd * Tm.f;                   // Dnn_(0, tmax)
      L.Tn = L.Dnn * opn;
    }
    L.Tt = cT * To.d * C.N0.f;                        // Tt_(0, opt)
    double Tt_d = L.Tt, e;
    if (opt == 0.0) Tt_d = icf_law_zero(C.gam_t, delt, C.zT, C.N0, e);
    else e = icf_law_bound(cT, To, C.N0);
    if (icf_near(Tt_d, e, eps_neg) || (t_past && icf_near(Tt_d, e, thr_t))) {
      if (EXACT) Tt_d = icf_law_exact_T(C, deln, delt, 0.0, opt).y;
      else undecided = true;
    }
    if (Tt_d >= eps_neg && !(t_past && Tt_d < thr_t)) {
      if (opt >= tmax) {
        tmax = opt;
        L.Dtt = cTT * To.dd * C.N0.f;                 // Dtt_(0, opt)
      } else {
        const double peak = cT * Tm.d * C.N0.f;       // Tt_(0, tmax)
        L.Tt = peak * opt / tmax;
        L.Dtt = peak / tmax;
      }
    } else {
      L.Tt = L.Dtt = L.Dnt = 0;
      L.Tn = L.Dnn = 0;
      L.failed = true;
    }
    return L;
  }
  const icf_axis No = icf_axis_eval(C.alpha, C.p_m, C.gam_n, C.pMnt, opn * ideln, C.alpha_int);
  L.Tt = cT * To.d * No.f;                            // Tt_(opn, opt)
  L.Tn = cN * No.d * To.f;                            // Tn_(opn, opt)
  const bool n_past = opn > deln * C.rn / 5;
  double Tt_d = L.Tt, Tn_d = L.Tn, et, en;
  if (opt == 0.0) Tt_d = icf_law_zero(C.gam_t, delt, C.zT, No, et);
  else et = icf_law_bound(cT, To, No);
  if (opn == 0.0) Tn_d = icf_law_zero(C.gam_n, deln, C.zN, To, en);
  else en = icf_law_bound(cN, No, To);
  if (icf_near(Tt_d, et, eps_neg) || icf_near(Tn_d, en, eps_neg) || (t_past && icf_near(Tt_d, et, thr_t)) ||
      (n_past && icf_near(Tn_d, en, thr_n))) {
    if (EXACT) {
      const double2 x = icf_law_exact_T(C, deln, delt, opn, opt);
      Tn_d = x.x;
      Tt_d = x.y;
    } else {
      undecided = true;
    }
  }
  if (Tt_d >= eps_neg && Tn_d >= eps_neg && !(t_past && Tt_d < thr_t) && !(n_past && Tn_d < thr_n)) {
    const bool tsoft = (opt >= tmax), nsoft = (opn >= pmax);
    if (tsoft && nsoft) {
      tmax = opt;
      pmax = opn;
      L.Dnn = cNN * No.dd * To.f;
      L.Dnt = cNT * No.d * To.d;
      L.Dtt = cTT * To.dd * No.f;
    } else if (tsoft && !nsoft) {
      if (pmax != 0) {
        const double peak = cN * Np.d * Tm.f;         // Tn_(pmax, tmax)
        L.Tn = peak * opn / pmax;
        L.Dnn = peak / pmax;
      } else {
        L.Tn = 0;
        L.Dnn = cNN * C.N0.dd * Tm.f;                 // Dnn_(0, tmax)
      }
      tmax = opt;
      L.Tt = cT * To.d * Np.f;                        // Tt_(pmax, opt)
      L.Dtt = cTT * To.dd * Np.f;                     // Dtt_(pmax, opt)
    } else if (!tsoft && nsoft) {
      if (tmax != 0) {
        const double peak = cT * Tm.d * Np.f;         // Tt_(pmax, tmax)
        L.Tt = peak * opt / tmax;
        L.Dtt = peak / tmax;
      } else {
        L.Tt = 0;
        L.Dtt = cTT * C.T0.dd * Np.f;                 // Dtt_(pmax, 0)
      }
      pmax = opn;
      L.Tn = cN * No.d * Tm.f;                        // Tn_(opn, tmax)
      L.Dnn = cNN * No.dd * Tm.f;                     // Dnn_(opn, tmax)
    } else {
      const double peakN = cN * Np.d * Tm.f;          // Tn_(pmax, tmax)
      if (pmax != 0) {
        L.Tn = peakN * opn / pmax;
        L.Dnn = peakN / pmax;
      } else {
        L.Tn = 0;
        L.Dnn = cNN * C.N0.dd * Tm.f;                 // Dnn_(0, tmax)
      }
      if (tmax != 0) {
        const double peakT = cT * Tm.d * Np.f;        // Tt_(pmax, tmax)
        L.Tt = peakT * opt / tmax;
        L.Dtt = peakT / tmax;
      } else {
        L.Tt = 0;
        L.Dtt = cTT * C.T0.dd * Np.f;                 // Dtt_(pmax, 0)
      }
    }
  } else {
    L.failed = true;
    L.Tn = L.Tt = L.Dnn = L.Dtt = L.Dnt = 0;
  }
  return L;
}
