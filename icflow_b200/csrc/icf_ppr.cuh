// icf_ppr.cuh -- Park-Paulino-Roesler cohesive law on the device.
//
// PPR potential derivatives (cz_kernels9/PPR_math.h:2-57) and the
// thermodynamically consistent law with unload/reload and contact branches
// (cz_kernels9/cz_kernels.h:37-174).  The branch structure is the algorithm
// and is kept; the power factors of one axis are evaluated once per call and
// shared between the traction and tangent that use them.
#pragma once
#include <cuda_runtime.h>

struct icf_ppr_c {
  double alpha, beta, p_m, p_n, deln, delt, gam_n, gam_t, pMtn, pMnt;
  double rn, rt, f_tn, f_tt;
};

// (1-x)^(a-k) and (p/a + x)^(p-k) for k = 0, 1, 2.
struct icf_pw {
  double o0, o1, o2, s0, s1, s2;
};

__device__ __forceinline__ icf_pw icf_pows(double a, double p, double x) {
  icf_pw w;
  const double o = 1.0 - x, s = (p / a) + x;
  w.o0 = pow(o, a);
  w.o1 = pow(o, a - 1.0);
  w.o2 = pow(o, a - 2.0);
  w.s0 = pow(s, p);
  w.s1 = pow(s, p - 1.0);
  w.s2 = pow(s, p - 2.0);
  return w;
}

// Values of the five PPR functions at one (dn, dt), sharing the power
// factors: Tn, Tt, Dnn, Dtt, Dnt.
struct icf_ppr_v {
  double Tn, Tt, Dnn, Dtt, Dnt;
};

__device__ __forceinline__ icf_ppr_v icf_ppr_all(const icf_ppr_c &q, double dn,
                                                 double dt) {
  const icf_pw N = icf_pows(q.alpha, q.p_m, dn / q.deln);
  const icf_pw T = icf_pows(q.beta, q.p_n, dt / q.delt);
  const double a = q.alpha, pm = q.p_m, b = q.beta, pn = q.p_n;
  const double dN = (pm * N.o0 * N.s1) - (a * N.o1 * N.s0);
  const double dT = pn * T.o0 * T.s1 - b * T.o1 * T.s0;
  const double fN = q.gam_n * N.o0 * N.s0 + q.pMnt;
  const double fT = q.gam_t * T.o0 * T.s0 + q.pMtn;
  const double ddN = (pm * pm - pm) * N.o0 * N.s2 + (a * a - a) * N.o2 * N.s0 -
                     2.0 * a * pm * N.o1 * N.s1;
  const double ddT = (pn * pn - pn) * T.o0 * T.s2 + (b * b - b) * T.o2 * T.s0 -
                     2.0 * b * pn * T.o1 * T.s1;
  icf_ppr_v v;
  v.Tn = (q.gam_n / q.deln) * dN * fT;
  v.Tt = (q.gam_t / q.delt) * dT * fN;
  v.Dnn = (q.gam_n / (q.deln * q.deln)) * ddN * fT;
  v.Dtt = (q.gam_t / (q.delt * q.delt)) * ddT * fN;
  v.Dnt = (q.gam_n * q.gam_t / (q.deln * q.delt)) * dN * dT;
  return v;
}

// Single functions (the law evaluates them at different arguments).
__device__ __forceinline__ double icf_ppr_Tn(const icf_ppr_c &q, double dn,
                                             double dt) {
  const icf_pw N = icf_pows(q.alpha, q.p_m, dn / q.deln);
  const icf_pw T = icf_pows(q.beta, q.p_n, dt / q.delt);
  const double dN = (q.p_m * N.o0 * N.s1) - (q.alpha * N.o1 * N.s0);
  return (q.gam_n / q.deln) * dN * (q.gam_t * T.o0 * T.s0 + q.pMtn);
}
__device__ __forceinline__ double icf_ppr_Tt(const icf_ppr_c &q, double dn,
                                             double dt) {
  const icf_pw N = icf_pows(q.alpha, q.p_m, dn / q.deln);
  const icf_pw T = icf_pows(q.beta, q.p_n, dt / q.delt);
  const double dT = q.p_n * T.o0 * T.s1 - q.beta * T.o1 * T.s0;
  return (q.gam_t / q.delt) * dT * (q.gam_n * N.o0 * N.s0 + q.pMnt);
}
__device__ __forceinline__ double icf_ppr_Dnn(const icf_ppr_c &q, double dn,
                                              double dt) {
  const icf_pw N = icf_pows(q.alpha, q.p_m, dn / q.deln);
  const icf_pw T = icf_pows(q.beta, q.p_n, dt / q.delt);
  const double a = q.alpha, pm = q.p_m;
  const double ddN = (pm * pm - pm) * N.o0 * N.s2 + (a * a - a) * N.o2 * N.s0 -
                     2.0 * a * pm * N.o1 * N.s1;
  return (q.gam_n / (q.deln * q.deln)) * ddN * (q.gam_t * T.o0 * T.s0 + q.pMtn);
}
__device__ __forceinline__ double icf_ppr_Dtt(const icf_ppr_c &q, double dn,
                                              double dt) {
  const icf_pw N = icf_pows(q.alpha, q.p_m, dn / q.deln);
  const icf_pw T = icf_pows(q.beta, q.p_n, dt / q.delt);
  const double b = q.beta, pn = q.p_n;
  const double ddT = (pn * pn - pn) * T.o0 * T.s2 + (b * b - b) * T.o2 * T.s0 -
                     2.0 * b * pn * T.o1 * T.s1;
  return (q.gam_t / (q.delt * q.delt)) * ddT * (q.gam_n * N.o0 * N.s0 + q.pMnt);
}

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
    o0 = pow(o, a);
    o1 = o0 / o;
    o2 = o1 / o;
  } else {
    o0 = pow(o, a);
    o1 = pow(o, a - 1.0);
    o2 = pow(o, a - 2.0);
  }
  const double s0 = pow(s, p), s1 = s0 / s, s2 = s1 / s;
  icf_axis r;
  r.f = gam * o0 * s0 + mac;
  r.d = (p * o0 * s1) - (a * o1 * s0);
  r.dd = (p * p - p) * o0 * s2 + (a * a - a) * o2 * s0 - 2.0 * a * p * o1 * s1;
  return r;
}

struct icf_law_c {
  double alpha, beta, p_m, p_n, gam_n, gam_t, pMtn, pMnt, rn, rt;
  icf_axis N0, T0;  // axes at zero opening
  int alpha_int, beta_int;  // alpha, beta when they are integers in [2, 16], else 0
};

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
// tmax are updated in place.
__device__ inline icf_law icf_cz_law_hist(const icf_law_c &C, double f_tn, double f_tt, double deln,
                                          double delt, const icf_axis &Np, const icf_axis &Tm, double &pmax,
                                          double &tmax, double opn, double opt) {
  icf_law L;
  L.Tn = L.Tt = L.Dnn = L.Dtt = L.Dnt = 0;
  L.contact = false;
  L.failed = false;
  if (opn > deln || opt > delt) {
    L.failed = true;
    return L;
  }
  const double cN = C.gam_n / deln, cT = C.gam_t / delt;
  const double cNN = C.gam_n / (deln * deln), cTT = C.gam_t / (delt * delt);
  const double cNT = C.gam_n * C.gam_t / (deln * delt);
  L.contact = (opn < 0);
  const double eps_neg = -1e-9;
  const double thr_t = f_tt * 0.05, thr_n = f_tn * 0.05;
  const icf_axis To = icf_axis_eval(C.beta, C.p_n, C.gam_t, C.pMtn, opt / delt, C.beta_int);
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
    if (L.Tt >= eps_neg && !(opt > delt * C.rt / 5 && L.Tt < thr_t)) {
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
  const icf_axis No = icf_axis_eval(C.alpha, C.p_m, C.gam_n, C.pMnt, opn / deln, C.alpha_int);
  L.Tt = cT * To.d * No.f;                            // Tt_(opn, opt)
  L.Tn = cN * No.d * To.f;                            // Tn_(opn, opt)
  if (L.Tt >= eps_neg && L.Tn >= eps_neg && !(opt > delt * C.rt / 5 && L.Tt < thr_t) &&
      !(opn > deln * C.rn / 5 && L.Tn < thr_n)) {
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

// The same, evaluating the history axes itself.
__device__ inline icf_law icf_cz_law_axes(const icf_law_c &C, double f_tn, double f_tt,
                                          double deln, double delt, double &pmax,
                                          double &tmax, double opn, double opt) {
  icf_axis Np, Tm;
  icf_cz_hist_axes(C, deln, delt, pmax, tmax, Np, Tm);
  return icf_cz_law_hist(C, f_tn, f_tt, deln, delt, Np, Tm, pmax, tmax, opn, opt);
}

// cohesive_law_thermodynamically_consistent (cz_kernels.h:37-174); pmax and
// tmax are updated in place.
__device__ inline icf_law icf_cz_law(const icf_ppr_c &q, double &pmax,
                                     double &tmax, double opn, double opt) {
  icf_law L;
  L.Tn = L.Tt = L.Dnn = L.Dtt = L.Dnt = 0;
  L.contact = false;
  L.failed = false;
  if (opn > q.deln || opt > q.delt) {
    L.failed = true;
    return L;
  }
  L.contact = (opn < 0);
  const double eps_neg = -1e-9;
  const double thr_t = q.f_tt * 0.05, thr_n = q.f_tn * 0.05;
  if (L.contact) {
    if (pmax != 0) {
      const double peak = icf_ppr_Tn(q, pmax, tmax);
      L.Tn = peak * opn / pmax;
      L.Dnn = peak / pmax;
    } else {
      L.Dnn = icf_ppr_Dnn(q, 0, tmax);
      L.Tn = L.Dnn * opn;
    }
    L.Tt = icf_ppr_Tt(q, 0, opt);
    if (L.Tt >= eps_neg && !(opt > q.delt * q.rt / 5 && L.Tt < thr_t)) {
      if (opt >= tmax) {
        tmax = opt;
        L.Dtt = icf_ppr_Dtt(q, 0, opt);
      } else {
        const double peak = icf_ppr_Tt(q, 0, tmax);
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
  // not in contact: both tractions at the current opening
  const icf_ppr_v cur = icf_ppr_all(q, opn, opt);
  L.Tt = cur.Tt;
  L.Tn = cur.Tn;
  if (L.Tt >= eps_neg && L.Tn >= eps_neg &&
      !(opt > q.delt * q.rt / 5 && L.Tt < thr_t) &&
      !(opn > q.deln * q.rn / 5 && L.Tn < thr_n)) {
    const bool tsoft = (opt >= tmax), nsoft = (opn >= pmax);
    if (tsoft && nsoft) {
      tmax = opt;
      pmax = opn;
      L.Dnn = cur.Dnn;
      L.Dnt = cur.Dnt;
      L.Dtt = cur.Dtt;
    } else if (tsoft && !nsoft) {
      if (pmax != 0) {
        const double peak = icf_ppr_Tn(q, pmax, tmax);
        L.Tn = peak * opn / pmax;
        L.Dnn = peak / pmax;
      } else {
        L.Tn = 0;
        L.Dnn = icf_ppr_Dnn(q, 0, tmax);
      }
      tmax = opt;
      L.Tt = icf_ppr_Tt(q, pmax, opt);
      L.Dtt = icf_ppr_Dtt(q, pmax, opt);
    } else if (!tsoft && nsoft) {
      if (tmax != 0) {
        const double peak = icf_ppr_Tt(q, pmax, tmax);
        L.Tt = peak * opt / tmax;
        L.Dtt = peak / tmax;
      } else {
        L.Tt = 0;
        L.Dtt = icf_ppr_Dtt(q, pmax, 0);
      }
      pmax = opn;
      L.Tn = icf_ppr_Tn(q, pmax, tmax);
      L.Dnn = icf_ppr_Dnn(q, pmax, tmax);
    } else {
      const double peakN = icf_ppr_Tn(q, pmax, tmax);
      if (pmax != 0) {
        L.Tn = peakN * opn / pmax;
        L.Dnn = peakN / pmax;
      } else {
        L.Tn = 0;
        L.Dnn = icf_ppr_Dnn(q, 0, tmax);
      }
      if (tmax != 0) {
        const double peakT = icf_ppr_Tt(q, pmax, tmax);
        L.Tt = peakT * opt / tmax;
        L.Dtt = peakT / tmax;
      } else {
        L.Tt = 0;
        L.Dtt = icf_ppr_Dtt(q, pmax, 0);
      }
    }
  } else {
    L.failed = true;
    L.Tn = L.Tt = L.Dnn = L.Dtt = L.Dnt = 0;
  }
  return L;
}
