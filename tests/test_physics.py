"""Physics invariants of the oracle, independent of the reference code:
zero elastic force under rigid motion, finite-difference consistency of the
element tangent, of the point-triangle derivatives in every region, and of the
PPR tractions and tangents."""
import numpy as np
import pytest

from oracle.oracle import Oracle

PRMS = dict(Y=9e9, nu=0.3, rho=916.0, phi_n=3.0, phi_t=3.0, sigma_max=1e6, tau_max=1e6,
            alpha=4.0, beta=4.0, lambda_n=0.02, lambda_t=0.02)


@pytest.fixture(scope="module")
def O():
    return Oracle()


@pytest.fixture(scope="module")
def p(O):
    return O.prms(**PRMS)


def _unit_tet():
    return np.array([0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 1], float) * 0.1


def test_rigid_motion_gives_no_force(O, p):
    x0 = _unit_tet()
    f, Df, V = O.elem_F_Df(p, x0, np.zeros(12))
    assert abs(V - 0.1 ** 3 / 6) < 1e-18 and np.abs(f).max() == 0
    c = x0.reshape(4, 3)
    th = 0.7
    R = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1]])
    un = ((c @ R.T) + np.array([0.3, -0.2, 0.1]) - c).ravel()
    f, Df, _ = O.elem_F_Df(p, x0, un)
    assert np.abs(f).max() <= 1e-6 * np.abs(Df).max() * 1e-1
    K0 = O.elem_F_Df(p, x0, np.zeros(12))[1]
    # Df is R K R^T: same eigenvalues as K, symmetric positive semi-definite
    assert np.allclose(np.linalg.eigvalsh(Df), np.linalg.eigvalsh(K0), rtol=1e-10, atol=1e-3)
    assert np.allclose(Df, Df.T, rtol=0, atol=1e-6 * np.abs(Df).max())


def test_small_strain_tangent_matches_finite_difference(O, p):
    rng = np.random.default_rng(0)
    x0 = _unit_tet()
    un = (rng.random(12) - 0.5) * 1e-4
    f0, Df, _ = O.elem_F_Df(p, x0, un)
    eps = 1e-9
    J = np.zeros((12, 12))
    for j in range(12):
        d = np.zeros(12)
        d[j] = eps
        J[:, j] = (O.elem_F_Df(p, x0, un + d)[0] - O.elem_F_Df(p, x0, un - d)[0]) / (2 * eps)
    # the corotational tangent drops the rotation-derivative term: agreement at small strain
    assert np.abs(J - Df).max() <= 2e-3 * np.abs(Df).max()


def test_point_triangle_derivatives_by_region(O):
    rng = np.random.default_rng(1)
    seen = set()
    for x in rng.random((400, 12)):
        d, fd, sd, s, t, br = O.pt(x)
        h = 1e-6
        g = np.zeros(12)
        H = np.zeros((12, 12))
        ok = True
        for j in range(12):
            e = np.zeros(12)
            e[j] = h
            dp, fdp, _, _, _, bp = O.pt(x + e)
            dm, fdm, _, _, _, bm = O.pt(x - e)
            if bp != br or bm != br:
                ok = False
                break
            g[j] = (dp - dm) / (2 * h)
            H[:, j] = (fdp - fdm) / (2 * h)
        if not ok:
            continue
        seen.add(br)
        assert np.abs(g - fd).max() <= 1e-6 * max(1.0, np.abs(fd).max())
        assert np.abs(H - sd).max() <= 1e-4 * max(1.0, np.abs(sd).max())
    assert seen >= {0, 1, 2, 3, 4, 5, 6}


def test_ppr_tangents_match_finite_differences(O, p):
    q = p.ppr
    for dn, dt in [(0.1, 0.2), (0.3, 0.05), (0.6, 0.4), (0.05, 0.7)]:
        a = dn * q.deln
        b = dt * q.delt
        Tn, Tt, Dnn, Dtt, Dnt = O.ppr_eval(p, a, b)
        hn, ht = 1e-7 * q.deln, 1e-7 * q.delt
        dTn = (O.ppr_eval(p, a + hn, b)[0] - O.ppr_eval(p, a - hn, b)[0]) / (2 * hn)
        dTt = (O.ppr_eval(p, a, b + ht)[1] - O.ppr_eval(p, a, b - ht)[1]) / (2 * ht)
        dTnt = (O.ppr_eval(p, a, b + ht)[0] - O.ppr_eval(p, a, b - ht)[0]) / (2 * ht)
        assert abs(dTn - Dnn) <= 1e-5 * abs(Dnn)
        assert abs(dTt - Dtt) <= 1e-5 * abs(Dtt)
        assert abs(dTnt - Dnt) <= 1e-5 * abs(Dnt) + 1e-9 * abs(Dnn)
    # peak normal traction is the strength sigma_max at lambda_n * deln
    Tn_peak = O.ppr_eval(p, q.rn * q.deln, 0.0)[0]
    assert abs(Tn_peak / q.f_tn - 1) < 1e-9
