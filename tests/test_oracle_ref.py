"""The CPU oracle against the reference's own kernel sources built for the host
(oracle/_ref), on fresh seeded inputs, including the unmodified reference
kernels driven through their strided layouts.  Skipped where the reference
build is absent (it needs the reference sources at build time)."""
import numpy as np
import pytest

from oracle.oracle import Oracle, RefKernels, ref_available
from tests.harness import rowwise_rel, vec_rel

pytestmark = pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
PRMS = dict(Y=9e9, nu=0.3, rho=916.0, phi_n=3.0, phi_t=3.0, sigma_max=1e6, tau_max=1e6,
            alpha=4.0, beta=4.0, lambda_n=0.02, lambda_t=0.02, penaltyK=1e8)


@pytest.fixture(scope="module")
def env():
    O = Oracle()
    R = RefKernels(nthreads=2)
    p = O.prms(**PRMS)
    R.set_constants(p)
    return O, R, p


def test_elements_random_bitexact(env):
    O, R, p = env
    rng = np.random.default_rng(101)
    from icflow_b200 import mesh as M

    x0 = rng.random((300, 4, 3))
    V = M._jdet(x0)
    x0[V < 0] = x0[V < 0][:, [0, 1, 3, 2]]
    x0 = x0.reshape(300, 12)
    un = (rng.random((300, 12)) - 0.5) * 0.05
    f, Df, V = R.F_and_Df(x0, un)
    for i in range(300):
        a = O.elem_F_Df(p, x0[i], un[i])
        assert np.array_equal(a[0], f[i]) and np.array_equal(a[1], Df[i])


def test_law_random_bitexact(env):
    O, R, p = env
    q = p.ppr
    rng = np.random.default_rng(102)
    n = 3000
    pm = rng.random(n) * q.deln * (rng.random(n) > 0.25)
    tm = rng.random(n) * q.delt * (rng.random(n) > 0.25)
    opn = (rng.random(n) * 2.2 - 1.1) * q.deln
    opt = rng.random(n) * 1.1 * q.delt
    pm2, tm2, law, fl = R.cz_law(pm, tm, opn, opt)
    early = (opn > q.deln) | (opt > q.delt)
    for i in range(n):
        a = O.cz_law(p, pm[i], tm[i], opn[i], opt[i])
        lim = 5 if early[i] else 6  # Dtn is unset by the reference on the early-failure path
        assert np.array_equal(a[2][:lim], law[i][:lim]) and np.array_equal(a[3], fl[i])
        assert a[0] == pm2[i] and a[1] == tm2[i]


def test_pt_random(env):
    O, R, p = env
    rng = np.random.default_rng(103)
    for x in rng.random((1500, 12)):
        a, b = O.pt(x), R.pt(x)
        assert a[5] == b[5] and a[3] == b[3] and a[4] == b[4]
        assert abs(a[0] - b[0]) <= 1e-13 * b[0]
        assert np.abs(a[2] - b[2]).max() <= 1e-12 * np.abs(b[2]).max()


def test_full_kernels_through_reference_layouts(env):
    """kelElementElasticityForce, kczCZForce (per-CZ strengths) and
    kCollisionResponseForce, unmodified, against the oracle's assembly."""
    O, R, p = env
    from icflow_b200 import mesh as M

    c = M.polycrystal(n=6, grains=6, seed=5, platens=True, gap=-0.3)
    nn = len(c.x0)
    rng = np.random.default_rng(104)
    un = (rng.random((nn, 3)) - 0.5) * 2e-6
    un[c.anchored] = 0
    vn = rng.random((nn, 3)) - 0.5
    an = rng.random((nn, 3)) - 0.5
    xt = c.x0 + un
    pairs = M.candidate_pairs(c, xt)
    masks = O.narrow_phase(pairs, c.selem, xt)
    imps = O.impacts(pairs, masks, c.selem, c.adj_off, c.adj, c.faces, xt)
    N, rows, cols = O.build_structure(c.alt, c.elems, c.czs, imps)
    ep = O.pcsr(c.elems, 4, c.alt, rows, cols, N)
    cp = O.pcsr(c.czs, 6, c.alt, rows, cols, N)
    ipc = O.pcsr(imps, 4, c.alt, rows, cols, N)
    nc = len(c.czs)
    pmax = rng.random((nc, 3)) * p.ppr.deln * 0.3
    tmax = rng.random((nc, 3)) * p.ppr.delt * 0.3
    sig = M.lognormal_strengths(nc, seed=3, granule_pairs=c.meshes[0].cz_grains)
    qs = [O.ppr_for(p, s, s) for s in sig]
    h = 1e-5
    st = R.pack_nodes(c.x0, un, vn, an)
    vals = np.zeros(9 * len(cols))
    rhs = np.zeros(3 * N)
    R.elem_kernel(st, h, c.elems, ep, vals, rhs)
    per_cz = (sig, sig, np.array([q.deln for q in qs]), np.array([q.delt for q in qs]))
    tp, tt, fl, avg = R.cz_kernel(st, h, c.czs, cp, pmax, tmax, vals, rhs, per_cz=per_cz)
    R.collision_kernel(st, h, imps, ipc, vals, rhs, p.penaltyK, p.DistanceEpsilon)
    res = O.assemble(p, h, c.x0, un, vn, an, c.elems, ep, c.czs, cp, pmax, tmax, imps, ipc, len(cols), N,
                     cz_ppr=qs)
    assert rowwise_rel(rows, vals.reshape(-1, 3, 3), res["vals"]) <= 1e-12
    assert vec_rel(rhs, res["rhs"]) <= 1e-12
    assert np.array_equal(fl, res["flags"])
    assert np.array_equal(tp[:, 0], res["tent"][:, 0]) and np.array_equal(tt[:, 0], res["tent"][:, 1])
    assert vec_rel(R.node_field(st, 12, nn), res["nodeF"]) <= 1e-12
    # narrow phase and closest face through the reference kernels
    rm, ie, el_stride = R.narrow_phase_kernel(R.pack_nodes(c.x0, un, vn, an), nn, pairs, c.selem, c.adj_off,
                                              c.adj)
    assert np.array_equal(rm, masks)
    ref_imp = R.closest_face_kernel(st, imps[:, :1].repeat(2, 1) * 0 + np.array(
        sorted({(int(c.selem[b][k]), int(a)) for (a, b), m in zip(pairs, masks) for k in range(4) if m & (1 << k)}
               | {(int(c.selem[a][k]), int(b)) for (a, b), m in zip(pairs, masks) for k in range(4)
                  if m & (16 << k)}), np.int32), ie, el_stride, c.faces)
    assert np.array_equal(ref_imp, imps)
