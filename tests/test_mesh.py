"""Synthetic mesh generator: the conventions the assembly relies on."""
import numpy as np

from icflow_b200 import mesh as M


def test_cantilever_counts_and_conventions():
    c = M.cantilever()
    assert len(c.elems) == 2304 and len(c.czs) == 32
    assert len(c.x0) == 625 + 25  # mid-span nodes split once
    V = M._jdet(c.x0[c.elems]) / 6
    assert np.all(V > 0) and abs(V.sum() - 0.006) < 1e-12
    # CZ vertex i+3 is the copy of vertex i on the other grain
    assert np.allclose(c.x0[c.czs[:, :3]], c.x0[c.czs[:, 3:]])
    assert np.all(c.czs[:, :3] != c.czs[:, 3:])
    # alt ids number the active nodes in order; anchored nodes have -1
    act = np.nonzero(c.alt >= 0)[0]
    assert np.array_equal(c.alt[act], np.arange(len(act))) and np.all(c.alt[c.anchored] == -1)
    assert c.n_active == 600


def test_polycrystal_cz_faces_and_adjacency():
    c = M.polycrystal(n=6, grains=6, seed=3, platens=True)
    m = c.meshes[0]
    # each CZ's two faces are listed after the exposed faces, first face on vrts 0..2
    fa = m.faces[m.cz_faces[:, 0]]
    assert np.array_equal(np.sort(fa, 1), np.sort(m.czs[:, :3], 1))
    assert not m.face_exposed[m.cz_faces].any() and m.face_exposed[: m.cz_faces.min()].all()
    # nodes of different grains are never shared by a tet pair across a CZ
    g = m.granule
    for e0, e1 in zip(*np.nonzero(g[:, None] != g[None, :])[:2]) if len(g) < 50 else []:
        assert not set(m.elems[e0]) & set(m.elems[e1])
    # adjacent faces of a surface element touch one of its vertices, in order, no duplicates
    for i in range(0, len(c.selem), 97):
        faces = c.adj[c.adj_off[i]:c.adj_off[i + 1]]
        assert len(set(faces.tolist())) == len(faces)
        for f in faces:
            assert set(c.faces[f].tolist()) & set(c.selem[i].tolist())
    V = M._jdet(c.x0[c.elems]) / 6
    assert np.all(V > 0)


def test_candidate_pairs_overlap_share_no_node_and_cover_the_meshes():
    c = M.polycrystal(n=6, grains=4, seed=1, platens=True, gap=-0.3)
    rng = np.random.default_rng(0)
    xt = c.x0 + (rng.random(c.x0.shape) - 0.5) * 1e-6
    lo = xt[c.selem].min(1)
    hi = xt[c.selem].max(1)
    for same in (True, False):
        pr = M.candidate_pairs(c, xt, same_mesh=same)
        assert len(pr) > 0 and np.all(pr[:, 0] < pr[:, 1])
        assert np.all((lo[pr[:, 0]] <= hi[pr[:, 1]]) & (lo[pr[:, 1]] <= hi[pr[:, 0]]))
        assert not (c.selem[pr[:, 0]][:, :, None] == c.selem[pr[:, 1]][:, None, :]).any()
        cross = c.selem_mesh[pr[:, 0]] != c.selem_mesh[pr[:, 1]]
        assert cross.all() if not same else (~cross).any()
    # every pair of the cross-mesh list is in the full one
    full = set(map(tuple, M.candidate_pairs(c, xt).tolist()))
    assert all(tuple(p) in full for p in M.candidate_pairs(c, xt, same_mesh=False).tolist())


def test_lognormal_strengths():
    s = M.lognormal_strengths(20000, mean=1e6, cv=0.2, seed=0)
    assert abs(s.mean() / 1e6 - 1) < 0.01 and abs(s.std() / s.mean() - 0.2) < 0.01
