"""Cohesive-law test cases placed at the law's decision thresholds.

The reference law (cz_kernels9/cz_kernels.h:37-174) fails a Gauss point when
Tt_ or Tn_ (PPR_math.h:2-24) is below -1e-9, or below 5 % of the strength past
a fifth of the characteristic opening.  These helpers find, with the CPU
oracle, the adjacent doubles at which the oracle's failure flag flips, and
return states a few ulps either side of each flip:

  tangential 5 %: opt crossing, opn = 0, small or in contact (opn < 0)
  normal 5 %:     opn crossing, opt = 0 or small
  -1e-9 at zero opening: the strength at which the rounding noise of
                  Tt_(0, 0) / Tn_(0, 0) crosses -1e-9 (the noise scales with
                  the strength through 1/del)
  exact input comparisons: opt = del_t lambda_t / 5, opn = pmax, opt = tmax,
                  opn = del_n, opt = del_t, each +- 1 ulp

A flag computed from such a state is reproducible only with the same rounding
as the reference.  `pinned` tells, per state, whether the host C library's pow
(which the oracle, like the reference's host build, calls) is correctly
rounded on every pow the state's Tn_ and Tt_ evaluate; it is checked against a
60-digit decimal evaluation.  Where it is not, the library itself is off by an
ulp and no other implementation can be expected to reproduce its flag.
"""
from __future__ import annotations

import math
from decimal import Decimal, getcontext

import numpy as np

SIG = 1e6  # strength of the benchmark configurations


def correct_pow(x: float, y: float) -> float:
    """x**y correctly rounded to double (60 significant digits, then one
    rounding)."""
    if y == 0.0 or x == 1.0:
        return 1.0
    if x == 0.0:
        return 0.0 if y > 0 else math.inf
    getcontext().prec = 60
    return float((Decimal(y) * Decimal(x).ln()).exp())


def pow_args(q, opn: float, opt: float, contact: bool):
    """The (base, exponent) pairs of the pow calls Tn_ and Tt_ make at this
    state (PPR_math.h:2-24); in contact the law evaluates Tt_(0, opt) only."""
    dn = 0.0 if contact else opn
    xn = dn / q.deln
    xt = opt / q.delt
    sn = q.p_m / q.alpha + xn
    st = q.p_n / q.beta + xt
    return [(1.0 - xn, q.alpha), (1.0 - xn, q.alpha - 1.0), (sn, q.p_m - 1.0), (sn, q.p_m),
            (1.0 - xt, q.beta), (1.0 - xt, q.beta - 1.0), (st, q.p_n - 1.0), (st, q.p_n)]


def pinned(q, opn: float, opt: float) -> bool:
    if opn > q.deln or opt > q.delt:  # the law fails before any pow
        return True
    return all(math.pow(x, y) == correct_pow(x, y) for x, y in pow_args(q, opn, opt, opn < 0))


def _failed(O, p, q, pmax, tmax, opn, opt) -> int:
    return int(O.cz_law(p, pmax, tmax, opn, opt, q)[3][1])


def _flip(f, lo: float, hi: float) -> tuple[float, float] | None:
    """Adjacent doubles a < b with f(a) != f(b), given f(lo) != f(hi)."""
    flo = f(lo)
    if flo == f(hi):
        return None
    for _ in range(200):
        if np.nextafter(lo, hi) == hi:
            return lo, hi
        mid = 0.5 * (lo + hi)
        if mid <= lo or mid >= hi:
            mid = float(np.nextafter(lo, hi))
        if f(mid) == flo:
            lo = mid
        else:
            hi = mid
    return None


def _scan(f, a: float, b: float, n: int = 64):
    """All flips of f on [a, b], located to adjacent doubles."""
    xs = np.linspace(a, b, n)
    vals = [f(float(x)) for x in xs]
    out = []
    for i in range(n - 1):
        if vals[i] != vals[i + 1]:
            r = _flip(f, float(xs[i]), float(xs[i + 1]))
            if r:
                out.append(r)
    return out


def _around(v: float, k: int = 3):
    out = [v]
    lo = hi = v
    for _ in range(k):
        lo = float(np.nextafter(lo, -math.inf))
        hi = float(np.nextafter(hi, math.inf))
        out += [lo, hi]
    return out


def threshold_cases(O, p):
    """States (pmax, tmax, opn, opt, sigma) at the law's thresholds, each
    a few ulps either side of a flip of the oracle's failure flag."""
    cases = []
    q = p.ppr

    def add(pm, tm, opn, opt, sig=SIG):
        cases.append((pm, tm, opn, opt, sig))

    # tangential 5 % threshold past the peak, out of contact and in contact
    for opn_rel in (0.0, 1e-3, 0.01, -0.05):
        opn = opn_rel * q.deln
        for tm_rel in (0.0, 0.3):
            f = lambda o: _failed(O, p, q, 0.0, tm_rel * q.delt, opn, o)  # noqa: E731
            for a, b in _scan(f, q.delt * q.rt / 5 * 1.0001, q.delt * 0.99999):
                for o in _around(a) + _around(b):
                    add(0.0, tm_rel * q.delt, opn, o)
    # normal 5 % threshold
    for opt_rel in (0.0, 1e-3, 0.01):
        opt = opt_rel * q.delt
        for pm_rel in (0.0, 0.3):
            f = lambda o: _failed(O, p, q, pm_rel * q.deln, 0.0, o, opt)  # noqa: E731
            for a, b in _scan(f, q.deln * q.rn / 5 * 1.0001, q.deln * 0.99999):
                for o in _around(a) + _around(b):
                    add(pm_rel * q.deln, 0.0, o, opt)
    # -1e-9 at zero opening: the strength at which the noise crosses it
    for opn, opt in ((0.0, 0.0), (-1e-12, 0.0)):
        def fs(s, opn=opn, opt=opt):
            qs = O.ppr_for(p, s, s)
            return _failed(O, p, qs, 0.0, 0.0, opn, opt)
        for a, b in _scan(fs, 1e6, 4e7, 96)[:6]:
            for s in _around(a, 1) + _around(b, 1):
                add(0.0, 0.0, opn, opt, s)
    # zero openings at a range of strengths, both sides of the noise threshold
    for s in np.geomspace(5e5, 5e7, 25):
        for opn, opt in ((0.0, 0.0), (0.0, 1e-21), (1e-21, 0.0), (-1e-9, 0.0)):
            add(0.0, 0.0, opn, opt, float(s))
    # comparisons on the inputs themselves
    t5 = q.delt * q.rt / 5
    n5 = q.deln * q.rn / 5
    for o in _around(t5, 2):
        add(0.0, 0.0, 0.0, o)
    for o in _around(n5, 2):
        add(0.0, 0.0, o, 0.0)
    for pm in (0.2 * q.deln, 0.5 * q.deln):
        for o in _around(pm, 1):
            add(pm, 0.1 * q.delt, o, 0.05 * q.delt)
    for tm in (0.2 * q.delt, 0.5 * q.delt):
        for o in _around(tm, 1):
            add(0.1 * q.deln, tm, 0.05 * q.deln, o)
    for o in _around(q.deln, 1):
        add(0.0, 0.0, o, 0.0)
    for o in _around(q.delt, 1):
        add(0.0, 0.0, 0.0, o)
    # the damaged threshold pmax >= deln lambda (flagged by the CZ kernel)
    for o in _around(q.deln * q.rn, 1):
        add(0.0, 0.0, o, 0.0)
    return np.array(cases, dtype=np.float64)


def oracle_law(O, p, cases):
    """The oracle's law on each state: pmax', tmax', law[5], contact, failed."""
    n = len(cases)
    pm = np.zeros(n)
    tm = np.zeros(n)
    law = np.zeros((n, 5))
    fl = np.zeros((n, 2), np.int32)
    qcache = {}
    for i, (a, b, opn, opt, s) in enumerate(cases):
        if s not in qcache:
            qcache[s] = O.ppr_for(p, s, s)
        r = O.cz_law(p, a, b, opn, opt, qcache[s])
        pm[i], tm[i] = r[0], r[1]
        law[i] = r[2][:5]
        fl[i] = r[3]
    return pm, tm, law, fl
