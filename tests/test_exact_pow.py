"""icf_exact.cuh on the host: the correctly rounded pow and the reference-order
Tn_/Tt_ that settle the cohesive law's undecided failure tests.

The header is compiled here with g++ (no floating-point contraction, as on
the device where every operation is an explicitly rounded intrinsic) into a
small shared library in a temporary directory.
"""
from __future__ import annotations

import ctypes as C
import math
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from tests.harness import Oracle, orc_prms_from
from tests.law_cases import correct_pow, pinned

from icflow_b200.model_prms import config_prms

HDR = Path(__file__).resolve().parents[1] / "icflow_b200" / "csrc" / "icf_exact.cuh"
SHIM = r"""
#include "icf_exact.cuh"
extern "C" double x_pow(double x, double y) { return icf_pow_cr(x, y); }
extern "C" void x_T(const double *k, double deln, double delt, double dn, double dt, double *out) {
  const icf_ppr_k K{k[0], k[1], k[2], k[3], k[4], k[5], k[6], k[7]};
  out[0] = icf_ref_Tn(K, deln, delt, dn, dt);
  out[1] = icf_ref_Tt(K, deln, delt, dn, dt);
}
"""


@pytest.fixture(scope="module")
def xlib(tmp_path_factory):
    if not shutil.which("g++"):
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("exact")
    (d / "shim.cpp").write_text(SHIM)
    so = d / "libexact.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-I", str(HDR.parent),
                    str(d / "shim.cpp"), "-o", str(so)], check=True)
    L = C.CDLL(str(so))
    L.x_pow.restype = C.c_double
    L.x_pow.argtypes = [C.c_double, C.c_double]
    return L


def test_pow_is_correctly_rounded(xlib):
    rng = np.random.default_rng(5)
    p_m = 0.004807692307692308
    ys = [4.0, 3.0, p_m, p_m - 1.0, 2.5, -0.9, 1.7, 7.3]
    n = 0
    glibc_off = 0
    for i in range(1500):
        r = i % 4
        x = [rng.random() * 1.0012, 0.0012 + rng.random() * 1e-6, 1 - rng.random() * 1e-3, rng.random() * 4][r]
        if x <= 0:
            continue
        y = ys[i % len(ys)] if i % 5 else rng.random() * 20 - 10
        cr = correct_pow(x, y)
        assert xlib.x_pow(x, y) == cr, (x, y)
        glibc_off += math.pow(x, y) != cr
        n += 1
    # the host library is correctly rounded but for values near a midpoint
    assert glibc_off < 0.01 * n


def test_reference_order_T_matches_the_oracle(xlib):
    """icf_ref_Tn/icf_ref_Tt give the oracle's (the reference expressions with
    the host pow) Tn_ and Tt_ bit for bit wherever that pow rounds correctly."""
    O = Oracle()
    p = orc_prms_from(O, config_prms())
    q = p.ppr
    K = np.array([q.alpha, q.beta, q.p_m, q.p_n, q.gam_n, q.gam_t, q.pMtn, q.pMnt])
    rng = np.random.default_rng(6)
    out = np.zeros(2)
    checked = 0
    for i in range(3000):
        dn = [0.0, rng.random() * q.deln, rng.random() * 1e-6 * q.deln][i % 3]
        dt = [rng.random() * q.delt, 0.0, rng.random() * 1e-9 * q.delt][(i // 3) % 3]
        if not pinned(q, dn, dt):
            continue
        xlib.x_T(K.ctypes.data_as(C.POINTER(C.c_double)), C.c_double(q.deln), C.c_double(q.delt),
                 C.c_double(dn), C.c_double(dt), out.ctypes.data_as(C.POINTER(C.c_double)))
        ref = O.ppr_eval(p, dn, dt)
        assert out[0] == ref[0] and out[1] == ref[1], (dn, dt, out, ref[:2])
        checked += 1
    assert checked > 2900
