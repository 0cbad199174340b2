// icf_exact.cuh -- the cohesive law's decision values, rounded as the
// reference's expressions round them.
//
// The law (cz_kernels9/cz_kernels.h:37-174) fails a Gauss point when a
// traction falls below -1e-9 or below 5 % of the strength past the peak.
// Those comparisons are made on Tn_ and Tt_ (cz_kernels9/PPR_math.h:2-24),
// and at a zero opening Tn_/Tt_ are rounding noise of about 1e-10 against the
// -1e-9 threshold.  So a flag is only reproducible if the decision value is
// the same floating-point number the reference computes: the same operations
// in the same order, each rounded on its own, and `pow` correctly rounded
// (the host C library's pow, which the reference's host build uses, is
// correctly rounded except in cases rarer than 1 in 10^4).
//
// icf_pow_cr is written here from two series and double-double arithmetic
// (Dekker's exact product through fma, Knuth's two-sum):
//   ln x = k ln 2 + 2 atanh(t),  t = (m - 1)/(m + 1),  x = m 2^k, m in [1/sqrt2, sqrt2)
//   exp y = 2^n (e^(r/256))^256,  r = y - n ln 2,  e^z by its Taylor series
// Its result before the final rounding is accurate to about 2^-95 relative,
// so it is the correctly rounded pow unless the exact value lies within
// 2^-42 of an ulp of a rounding midpoint.
//
// The law itself runs on the fast axis form (icf_ppr.cuh).  Each decision
// value comes with a bound on |fast - reference|; only a comparison that the
// bound cannot settle recomputes the value here (icf_law_decide), which in
// practice means openings that are exactly zero.
#pragma once
#include <cmath>

#ifdef __CUDACC__
#define ICF_HD __host__ __device__ __forceinline__
#else
#define ICF_HD inline
#endif

// Separately rounded operations.  Host code that includes this header must be
// compiled without floating-point contraction (-ffp-contract=off).
#if defined(__CUDA_ARCH__)
ICF_HD double icf_rmul(double a, double b) { return __dmul_rn(a, b); }
ICF_HD double icf_radd(double a, double b) { return __dadd_rn(a, b); }
ICF_HD double icf_rsub(double a, double b) { return __dsub_rn(a, b); }
ICF_HD double icf_rdiv(double a, double b) { return __ddiv_rn(a, b); }
ICF_HD double icf_fma(double a, double b, double c) { return __fma_rn(a, b, c); }
#else
ICF_HD double icf_rmul(double a, double b) { return a * b; }
ICF_HD double icf_radd(double a, double b) { return a + b; }
ICF_HD double icf_rsub(double a, double b) { return a - b; }
ICF_HD double icf_rdiv(double a, double b) { return a / b; }
ICF_HD double icf_fma(double a, double b, double c) { return std::fma(a, b, c); }
#endif

struct icf_dd {
  double hi, lo;
};

ICF_HD icf_dd icf_two_sum(double a, double b) {
  const double s = icf_radd(a, b);
  const double bb = icf_rsub(s, a);
  const double e = icf_radd(icf_rsub(a, icf_rsub(s, bb)), icf_rsub(b, bb));
  return icf_dd{s, e};
}
ICF_HD icf_dd icf_fast_two_sum(double a, double b) {  // |a| >= |b|
  const double s = icf_radd(a, b);
  return icf_dd{s, icf_rsub(b, icf_rsub(s, a))};
}
ICF_HD icf_dd icf_two_prod(double a, double b) {
  const double p = icf_rmul(a, b);
  return icf_dd{p, icf_fma(a, b, -p)};
}
ICF_HD icf_dd icf_dd_add(icf_dd a, icf_dd b) {
  icf_dd s = icf_two_sum(a.hi, b.hi);
  const icf_dd t = icf_two_sum(a.lo, b.lo);
  s.lo = icf_radd(s.lo, t.hi);
  s = icf_fast_two_sum(s.hi, s.lo);
  s.lo = icf_radd(s.lo, t.lo);
  return icf_fast_two_sum(s.hi, s.lo);
}
ICF_HD icf_dd icf_dd_mul(icf_dd a, icf_dd b) {
  icf_dd p = icf_two_prod(a.hi, b.hi);
  p.lo = icf_radd(p.lo, icf_radd(icf_rmul(a.hi, b.lo), icf_rmul(a.lo, b.hi)));
  return icf_fast_two_sum(p.hi, p.lo);
}
ICF_HD icf_dd icf_dd_mul_d(icf_dd a, double b) {
  icf_dd p = icf_two_prod(a.hi, b);
  p.lo = icf_radd(p.lo, icf_rmul(a.lo, b));
  return icf_fast_two_sum(p.hi, p.lo);
}
// a / b for a double-double b: one Newton correction of the double quotient
ICF_HD icf_dd icf_dd_div(icf_dd a, icf_dd b) {
  const double q1 = icf_rdiv(a.hi, b.hi);
  const icf_dd r = icf_dd_add(a, icf_dd_mul_d(b, -q1));
  const double q2 = icf_rdiv(r.hi, b.hi);
  const icf_dd r2 = icf_dd_add(r, icf_dd_mul_d(b, -q2));
  const double q3 = icf_rdiv(r2.hi, b.hi);
  icf_dd q = icf_fast_two_sum(q1, q2);
  return icf_dd_add(q, icf_dd{q3, 0.0});
}
// 1/k for a small positive integer k, as a double-double
ICF_HD icf_dd icf_dd_recip_int(double k) {
  const double h = icf_rdiv(1.0, k);
  const double r = icf_fma(-h, k, 1.0);  // exact remainder 1 - h k
  return icf_dd{h, icf_rdiv(r, k)};
}

// ln 2 to 106 bits (the mathematical constant, split into two doubles)
#define ICF_LN2_HI 0x1.62e42fefa39efp-1
#define ICF_LN2_LO 0x1.abc9e3b39803fp-56

// ln x for finite x > 0, as a double-double
ICF_HD icf_dd icf_log_dd(double x) {
  int k;
  double m = std::frexp(x, &k);  // x = m 2^k, m in [1/2, 1)
  if (m < 0.70710678118654752) {
    m = icf_rmul(m, 2.0);
    k -= 1;
  }
  // t = (m - 1)/(m + 1): m - 1 is exact (Sterbenz), m + 1 as a double-double
  const icf_dd t = icf_dd_div(icf_dd{icf_rsub(m, 1.0), 0.0}, icf_two_sum(m, 1.0));
  const icf_dd u = icf_dd_mul(t, t);  // u <= 0.0295
  // S = sum_n u^n / (2n + 1): the terms from n = 9 on are below 2^-46 and
  // are summed in double, the first nine in double-double
  double tail = 0.0;
  for (int n = 24; n >= 9; n--) tail = icf_radd(icf_rmul(tail, u.hi), icf_rdiv(1.0, 2.0 * n + 1.0));
  icf_dd S{tail, 0.0};
  for (int n = 8; n >= 0; n--) S = icf_dd_add(icf_dd_mul(S, u), icf_dd_recip_int(2.0 * n + 1.0));
  icf_dd r = icf_dd_mul(icf_dd_mul_d(t, 2.0), S);
  if (k != 0) {
    const icf_dd kl = icf_dd_add(icf_two_prod((double)k, ICF_LN2_HI), icf_two_prod((double)k, ICF_LN2_LO));
    r = icf_dd_add(kl, r);
  }
  return r;
}

// exp y for a double-double y, rounded to double (|y| < 700)
ICF_HD double icf_exp_dd(icf_dd y) {
  if (y.hi > 709.0) return HUGE_VAL;
  if (y.hi < -700.0) return 0.0;
  const double n = std::rint(icf_rdiv(y.hi, ICF_LN2_HI));
  // r = y - n ln 2, |r| <= 0.35
  icf_dd r = icf_dd_add(y, icf_two_prod(-n, ICF_LN2_HI));
  r = icf_dd_add(r, icf_two_prod(-n, ICF_LN2_LO));
  // z = r / 256 (exact), e^z by Horner: 1 + z (1 + z/2 (1 + z/3 (...)))
  const icf_dd z{std::ldexp(r.hi, -8), std::ldexp(r.lo, -8)};
  icf_dd e{1.0, 0.0};
  for (int j = 11; j >= 1; j--) {
    e = icf_dd_mul(e, icf_dd_mul(z, icf_dd_recip_int((double)j)));
    e = icf_dd_add(e, icf_dd{1.0, 0.0});
  }
  for (int i = 0; i < 8; i++) e = icf_dd_mul(e, e);
  return std::ldexp(icf_radd(e.hi, e.lo), (int)n);
}

// x^y, correctly rounded (see the head of this file), for x >= 0 and finite y;
// the law only raises positive bases, or zero to a positive power.
ICF_HD double icf_pow_cr(double x, double y) {
  if (y == 0.0 || x == 1.0) return 1.0;
  if (x == 0.0) return y > 0 ? 0.0 : HUGE_VAL;
  if (!(x > 0.0)) return NAN;
  const icf_dd L = icf_log_dd(x);
  icf_dd Y = icf_two_prod(y, L.hi);
  Y.lo = icf_radd(Y.lo, icf_rmul(y, L.lo));
  return icf_exp_dd(icf_fast_two_sum(Y.hi, Y.lo));
}

// The PPR constants the reference expressions read (cz_constants.h:6-14).
struct icf_ppr_k {
  double alpha, beta, p_m, p_n, gam_n, gam_t, pMtn, pMnt;
};

// Tn_ and Tt_ (PPR_math.h:2-24) in the reference's order of operations, each
// operation rounded on its own, pow correctly rounded.
ICF_HD double icf_ref_Tn(const icf_ppr_k &K, double deln, double delt, double Dn, double Dt) {
  const double Dndn = icf_rdiv(Dn, deln);
  const double Dtdt = icf_rdiv(Dt, delt);
  const double expr2 = icf_radd(icf_rdiv(K.p_m, K.alpha), Dndn);
  const double pr1 = icf_rdiv(K.gam_n, deln);
  const double on = icf_rsub(1.0, Dndn);
  const double pr2 = icf_rsub(icf_rmul(icf_rmul(K.p_m, icf_pow_cr(on, K.alpha)), icf_pow_cr(expr2, icf_rsub(K.p_m, 1.0))),
                              icf_rmul(icf_rmul(K.alpha, icf_pow_cr(on, icf_rsub(K.alpha, 1.0))), icf_pow_cr(expr2, K.p_m)));
  const double ot = icf_rsub(1.0, Dtdt);
  const double pr3 = icf_radd(icf_rmul(icf_rmul(K.gam_t, icf_pow_cr(ot, K.beta)),
                                       icf_pow_cr(icf_radd(icf_rdiv(K.p_n, K.beta), Dtdt), K.p_n)),
                              K.pMtn);
  return icf_rmul(icf_rmul(pr1, pr2), pr3);
}
ICF_HD double icf_ref_Tt(const icf_ppr_k &K, double deln, double delt, double Dn, double Dt) {
  const double Dndn = icf_rdiv(Dn, deln);
  const double Dtdt = icf_rdiv(Dt, delt);
  const double expr1 = icf_rsub(1.0, Dtdt);
  const double expr2 = icf_radd(icf_rdiv(K.p_n, K.beta), Dtdt);
  const double pr1 = icf_rdiv(K.gam_t, delt);
  const double pr2 = icf_rsub(icf_rmul(icf_rmul(K.p_n, icf_pow_cr(expr1, K.beta)), icf_pow_cr(expr2, icf_rsub(K.p_n, 1.0))),
                              icf_rmul(icf_rmul(K.beta, icf_pow_cr(expr1, icf_rsub(K.beta, 1.0))), icf_pow_cr(expr2, K.p_n)));
  const double on = icf_rsub(1.0, Dndn);
  const double pr3 = icf_radd(icf_rmul(icf_rmul(K.gam_n, icf_pow_cr(on, K.alpha)),
                                       icf_pow_cr(icf_radd(icf_rdiv(K.p_m, K.alpha), Dndn), K.p_m)),
                              K.pMnt);
  return icf_rmul(icf_rmul(pr1, pr2), pr3);
}
