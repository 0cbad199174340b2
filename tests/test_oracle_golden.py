"""The CPU oracle against golden fixtures produced by the reference's own kernel
code (tests/golden/make_golden.py).  Runs anywhere, no GPU, no reference
sources needed.  Element, PPR and law outputs are bit-identical to the
reference build; the point-triangle derivatives agree to 1e-12 (they are
evaluated through a different but equivalent chain of expressions)."""
from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import Oracle
from tests.harness import rowwise_rel, vec_rel

G = Path(__file__).resolve().parent / "golden"
PRMS = dict(Y=9e9, nu=0.3, rho=916.0, phi_n=3.0, phi_t=3.0, sigma_max=1e6, tau_max=1e6,
            alpha=4.0, beta=4.0, lambda_n=0.02, lambda_t=0.02, penaltyK=1e8)


@pytest.fixture(scope="module")
def O():
    return Oracle()


@pytest.fixture(scope="module")
def p(O):
    return O.prms(**PRMS)


def test_elem_bitexact(O, p):
    g = np.load(G / "elem_f_df.npz")
    for i in range(len(g["x0"])):
        f, Df, V = O.elem_F_Df(p, g["x0"][i], g["un"][i])
        assert np.array_equal(f, g["f"][i]) and np.array_equal(Df, g["Df"][i]) and V == g["V"][i], i


def test_ppr_and_law_bitexact(O, p):
    g = np.load(G / "cz_law.npz")
    for i in range(len(g["dn"])):
        assert np.array_equal(O.ppr_eval(p, g["dn"][i], g["dt"][i]), g["ppr"][i])
    for i in range(len(g["opn"])):
        pm, tm, law, fl = O.cz_law(p, g["pmax"][i], g["tmax"][i], g["opn"][i], g["opt"][i])
        ref = g["law"][i]
        keep = ~np.isnan(ref)
        assert np.array_equal(law[keep], ref[keep]), i
        assert np.array_equal(fl, g["flags"][i]) and pm == g["pmax_out"][i] and tm == g["tmax_out"][i]
    # every branch of the law is exercised by the fixture
    flags = g["flags"]
    assert flags[:, 0].any() and flags[:, 1].any() and (~flags.any(axis=1)).any()


def test_point_triangle(O):
    g = np.load(G / "pt.npz")
    seen = set()
    for i in range(len(g["x"])):
        d, fd, sd, s, t, br = O.pt(g["x"][i])
        assert br == g["branch"][i]
        seen.add(br)
        assert abs(d - g["dsq"][i]) <= 1e-13 * abs(g["dsq"][i])
        assert s == g["s"][i] and t == g["t"][i]
        assert np.abs(fd - g["fd"][i]).max() <= 1e-12 * np.abs(g["fd"][i]).max()
        assert np.abs(sd - g["sd"][i]).max() <= 1e-12 * np.abs(g["sd"][i]).max()
    assert seen == set(range(8)), seen
    h = np.load(G / "dtn.npz")
    for x, d in zip(h["x"], h["d"]):
        assert O.dtn(x[:9], x[9:]) == d


def test_cantilever_assembly(O, p):
    from icflow_b200 import mesh as M

    g = np.load(G / "cantilever_assembly.npz")
    c = M.cantilever()
    N, rows, cols = O.build_structure(c.alt, c.elems, c.czs, np.zeros((0, 4), np.int32))
    assert N == int(g["N"]) and np.array_equal(rows, g["rows"]) and np.array_equal(cols, g["cols"])
    ep = O.pcsr(c.elems, 4, c.alt, rows, cols, N)
    cp = O.pcsr(c.czs, 6, c.alt, rows, cols, N)
    res = O.assemble(p, float(g["h"]), c.x0, g["un"], g["vn"], g["an"], c.elems, ep, c.czs, cp, g["pmax"],
                     g["tmax"], np.zeros((0, 4), np.int32), np.zeros((0, 20), np.int32), len(cols), N)
    assert rowwise_rel(rows, g["vals"].reshape(-1, 3, 3), res["vals"]) <= 1e-12
    assert vec_rel(g["rhs"], res["rhs"]) <= 1e-12
    assert vec_rel(g["nodeF"], res["nodeF"]) <= 1e-12
    assert np.array_equal(res["flags"], g["flags"])
    assert np.array_equal(res["tent"][:, 0], g["tent_pmax"][:, 0])
    assert np.array_equal(res["tent"][:, 1], g["tent_tmax"][:, 0])
    assert vec_rel(g["avg"], res["avg"]) <= 1e-12


def test_contact_pipeline(O, p):
    from icflow_b200 import mesh as M

    g = np.load(G / "contact.npz")
    c = M.polycrystal(n=5, grains=4, seed=2, platens=True, gap=-0.3)
    xt = c.x0 + g["un"]
    # the fixture's pairs are those of different meshes
    pairs = M.candidate_pairs(c, xt, same_mesh=False, vertex_in_box=False)
    assert np.array_equal(pairs, g["pairs"])
    masks = O.narrow_phase(pairs, c.selem, xt)
    assert np.array_equal(masks, g["masks"])
    imps = O.impacts(pairs, masks, c.selem, c.adj_off, c.adj, c.faces, xt)
    assert len(imps) > 0 and np.array_equal(imps, g["impacts"])
    N, rows, cols = O.build_structure(c.alt, c.elems, c.czs, imps)
    assert np.array_equal(rows, g["rows"]) and np.array_equal(cols, g["cols"])
    ipc = O.pcsr(imps, 4, c.alt, rows, cols, N)
    nn = len(c.x0)
    res = O.assemble(p, 1e-5, c.x0, g["un"], np.zeros((nn, 3)), np.zeros((nn, 3)), np.zeros((0, 4), np.int32),
                     np.zeros((0, 20), np.int32), np.zeros((0, 6), np.int32), np.zeros((0, 42), np.int32),
                     np.zeros((0, 3)), np.zeros((0, 3)), imps, ipc, len(cols), N)
    ref = g["vals"].reshape(-1, 3, 3)
    touched = np.abs(ref).reshape(len(ref), -1).max(axis=1) > 0
    assert touched.any()
    assert np.abs(res["vals"] - ref).max() <= 1e-12 * np.abs(ref).max()
    assert vec_rel(g["rhs"], res["rhs"]) <= 1e-12
