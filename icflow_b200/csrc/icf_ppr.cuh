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
