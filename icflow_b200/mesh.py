"""Synthetic meshes and the MeshCollection bookkeeping of icFlow.

icFlow loads its setups from external files; none ship with it.  This module
generates seeded equivalents with the same conventions:

* structured box meshes split into tetrahedra (six per hexahedron, all sharing
  the hexahedron's main diagonal, so neighbouring cells conform);
* Voronoi grains from seeded uniform sites, and cohesive zones inserted on every
  face between two grains by splitting the nodes on grain boundaries, one copy
  per grain (v3Library/Geometry/Tools/CZInsertionTool.cs:371-491);
* the tetrahedron face convention {3,1,2}, {0,3,2}, {0,1,3}, {1,0,2}
  (CZInsertionTool.cs:162-166), CZ vertices vrts[0..2] on the first element's
  face and vrts[3+i] the copy of vrts[i] on the second (:207-219), exposed faces
  listed before the two faces of every CZ (:440-471);
* MeshCollection.Prepare ordering of nodes and faces over meshes
  (MeshCollection.cs:26-65), anchored nodes and alt ids in allNodes order
  (ImplicitModel3.cs:62-73), surface elements and their ordered adjacent faces
  (Mesh.cs:665-678, Element.cs:15-20).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# face f of a tet: its three vertices (CZInsertionTool.cs:162-166)
FACE_CONV = np.array([[3, 1, 2], [0, 3, 2], [0, 1, 3], [1, 0, 2]], dtype=np.int64)


def _jdet(x: np.ndarray) -> np.ndarray:
    """Rest Jacobian determinant of tets x[..., 4, 3] (element_kernels2.h:38-48)."""
    d = lambda c, i, j: x[..., i, c] - x[..., j, c]  # noqa: E731
    return (d(0, 1, 0) * (d(1, 1, 2) * d(2, 2, 3) - d(1, 2, 3) * d(2, 1, 2))
            + d(0, 2, 1) * (d(1, 2, 3) * d(2, 0, 1) - d(1, 0, 1) * d(2, 2, 3))
            + d(0, 3, 2) * (d(1, 0, 1) * d(2, 1, 2) - d(1, 1, 2) * d(2, 0, 1)))


def box_tets(n: tuple[int, int, int], size: tuple[float, float, float],
             origin=(0.0, 0.0, 0.0)) -> tuple[np.ndarray, np.ndarray]:
    """Structured grid of n[0] x n[1] x n[2] hexahedra, 6 tets each."""
    nx, ny, nz = n
    xs = origin[0] + np.linspace(0.0, size[0], nx + 1)
    ys = origin[1] + np.linspace(0.0, size[1], ny + 1)
    zs = origin[2] + np.linspace(0.0, size[2], nz + 1)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    x0 = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    order = np.lexsort((i, j, k))  # x fastest, then y, then z
    i, j, k = i[order], j[order], k[order]

    def nid(a, b, c):
        return (i + a) + (nx + 1) * ((j + b) + (ny + 1) * (k + c))

    unit = np.eye(3, dtype=np.int64)
    tets = []
    for perm in ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)):
        p1 = unit[perm[0]]
        p2 = p1 + unit[perm[1]]
        tets.append(np.stack([nid(0, 0, 0), nid(*p1), nid(*p2), nid(1, 1, 1)], axis=1))
    el = np.stack(tets, axis=1).reshape(-1, 4)
    # positive rest volume (V = Jdet / 6 "supposed to be positive", Element.cs)
    neg = _jdet(x0[el]) < 0
    el[neg] = el[neg][:, [0, 1, 3, 2]]
    return x0, el


def _tet_faces(elems: np.ndarray) -> np.ndarray:
    """[ne, 4, 3] face vertex ids in the face convention."""
    return elems[:, FACE_CONV]


def _face_keys(f: np.ndarray) -> np.ndarray:
    s = np.sort(f, axis=-1).astype(np.int64)
    return (s[..., 0] << 42) | (s[..., 1] << 21) | s[..., 2]


@dataclass
class Mesh:
    """One mesh of a collection (v3Library/Geometry/Mesh/Mesh.cs)."""

    x0: np.ndarray                      # [n, 3]
    elems: np.ndarray                   # [ne, 4]
    faces: np.ndarray                   # [nf, 3]
    face_exposed: np.ndarray            # [nf] bool
    czs: np.ndarray = field(default_factory=lambda: np.zeros((0, 6), np.int64))
    cz_faces: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), np.int64))
    granule: np.ndarray | None = None   # [ne]
    isDeformable: bool = True
    anchored: np.ndarray | None = None  # [n] bool, anchored surface nodes
    # prescribed motion of anchored surfaces: (node mask, dx, dy, dz, applicationTime)
    forced: list = field(default_factory=list)
    # rigid translation velocity for non-deformable meshes (TranslationCollection)
    velocity: tuple = (0.0, 0.0, 0.0)
    name: str = ""

    @property
    def n_nodes(self) -> int:
        return len(self.x0)


def box_mesh(n, size, origin=(0.0, 0.0, 0.0), deformable=True, name="") -> Mesh:
    x0, el = box_tets(n, size, origin)
    tf = _tet_faces(el).reshape(-1, 3)
    keys = _face_keys(tf)
    _, inv, cnt = np.unique(keys, return_inverse=True, return_counts=True)
    boundary = cnt[inv] == 1
    faces = tf[boundary]
    return Mesh(x0=x0, elems=el, faces=faces, face_exposed=np.ones(len(faces), bool),
                isDeformable=deformable, name=name)


def voronoi_grains(x0: np.ndarray, elems: np.ndarray, n_grains: int, seed: int,
                   lo=None, hi=None) -> np.ndarray:
    """Grain of every tet: the nearest of n_grains seeded uniform sites."""
    from scipy.spatial import cKDTree

    lo = x0.min(0) if lo is None else np.asarray(lo)
    hi = x0.max(0) if hi is None else np.asarray(hi)
    rng = np.random.default_rng(seed)
    sites = lo + rng.random((n_grains, 3)) * (hi - lo)
    cent = x0[elems].mean(axis=1)
    _, g = cKDTree(sites).query(cent)
    return g.astype(np.int64)


def insert_czs(m: Mesh, granule: np.ndarray) -> Mesh:
    """Cohesive zones on every face between two grains, with node splitting."""
    el = m.elems
    ne = len(el)
    tf = _tet_faces(el)                                  # [ne, 4, 3]
    keys = _face_keys(tf.reshape(-1, 3))
    order = np.argsort(keys, kind="stable")
    sk = keys[order]
    same = sk[1:] == sk[:-1]
    a_idx = order[:-1][same]                             # first occurrence (lower slot)
    b_idx = order[1:][same]
    ta, fa = a_idx // 4, a_idx % 4
    tb, fb = b_idx // 4, b_idx % 4
    swap = ta > tb                                        # e0 = lower tet index
    ta, tb = np.where(swap, tb, ta), np.where(swap, ta, tb)
    fa, fb = np.where(swap, fb, fa), np.where(swap, fa, fb)
    cz_sel = granule[ta] != granule[tb]
    ta, tb, fa, fb = ta[cz_sel], tb[cz_sel], fa[cz_sel], fb[cz_sel]
    order_cz = np.lexsort((fa, ta))
    ta, tb, fa, fb = ta[order_cz], tb[order_cz], fa[order_cz], fb[order_cz]

    # node copies, one per (node, grain) pair, numbered in node order then grain
    pairs = np.stack([el.ravel(), np.repeat(granule, 4)], axis=1)
    up, inv = np.unique(pairs, axis=0, return_inverse=True)
    inv = inv.ravel()
    new_el = inv.reshape(ne, 4)
    new_x0 = m.x0[up[:, 0]]
    G = int(granule.max()) + 1
    up_key = up[:, 0] * G + up[:, 1]          # ascending: np.unique sorts rows

    def copy_of(nodes, grains):
        return np.searchsorted(up_key, nodes * G + grains)

    face_a = el[ta[:, None], FACE_CONV[fa]]              # original ids, e0 convention
    face_b = el[tb[:, None], FACE_CONV[fb]]
    ga, gb = granule[ta], granule[tb]
    cz = np.empty((len(ta), 6), dtype=np.int64)
    for i in range(3):
        cz[:, i] = copy_of(face_a[:, i], ga)
        cz[:, 3 + i] = copy_of(face_a[:, i], gb)
    fa_new = new_el[ta[:, None], FACE_CONV[fa]]
    fb_new = new_el[tb[:, None], FACE_CONV[fb]]
    assert np.array_equal(np.sort(up[fb_new, 0], axis=1), np.sort(face_a, axis=1))
    assert np.array_equal(cz[:, :3], fa_new)

    # exposed faces of the split mesh (faces with one element), then CZ faces
    tfn = _tet_faces(new_el).reshape(-1, 3)
    kn = _face_keys(tfn)
    _, invn, cntn = np.unique(kn, return_inverse=True, return_counts=True)
    bnd = tfn[cntn[invn] == 1]
    cz_face_set = set(_face_keys(fa_new).tolist()) | set(_face_keys(fb_new).tolist())
    bk = _face_keys(bnd)
    exposed = bnd[~np.isin(bk, np.fromiter(cz_face_set, dtype=np.int64, count=len(cz_face_set)))]
    inner = np.empty((2 * len(cz), 3), dtype=np.int64)
    inner[0::2] = fa_new
    inner[1::2] = fb_new
    faces = np.concatenate([exposed, inner])
    face_exposed = np.concatenate([np.ones(len(exposed), bool), np.zeros(len(inner), bool)])
    ne_exp = len(exposed)
    cz_faces = np.stack([ne_exp + 2 * np.arange(len(cz)), ne_exp + 2 * np.arange(len(cz)) + 1], 1)
    out = Mesh(x0=new_x0, elems=new_el, faces=faces, face_exposed=face_exposed, czs=cz,
               cz_faces=cz_faces, granule=granule, isDeformable=True, name=m.name)
    out.cz_grains = np.stack([ga, gb], axis=1)
    return out


@dataclass
class Collection:
    """MeshCollection after Prepare/PrepareToCompute, as flat arrays."""

    meshes: list
    x0: np.ndarray = None            # allNodes rest coordinates [N, 3]
    anchored: np.ndarray = None      # [N] bool
    alt: np.ndarray = None           # [N] int32, -1 anchored
    elems: np.ndarray = None         # elasticElements [ne, 4] int32
    czs: np.ndarray = None           # allCZs of deformables [nc, 6] int32
    faces: np.ndarray = None         # allFaces [nf, 3] int32
    selem: np.ndarray = None         # surfaceElements [ns, 4] int32
    selem_mesh: np.ndarray = None    # mesh index of each surface element
    adj_off: np.ndarray = None       # [ns + 1] int32
    adj: np.ndarray = None           # adjacent faces of surface elements
    node_mesh: np.ndarray = None     # [N] mesh index
    n_active: int = 0

    def prepare(self):
        offs = np.cumsum([0] + [m.n_nodes for m in self.meshes])
        foffs = np.cumsum([0] + [len(m.faces) for m in self.meshes])
        self.x0 = np.concatenate([m.x0 for m in self.meshes]).astype(np.float64)
        self.node_mesh = np.concatenate([np.full(m.n_nodes, i) for i, m in enumerate(self.meshes)])
        anchored = np.zeros(len(self.x0), bool)
        for i, m in enumerate(self.meshes):
            if not m.isDeformable:
                anchored[offs[i]:offs[i + 1]] = True
            elif m.anchored is not None:
                anchored[offs[i]:offs[i + 1]] |= m.anchored
        self.anchored = anchored
        alt = np.full(len(self.x0), -1, np.int64)
        act = np.nonzero(~anchored)[0]
        alt[act] = np.arange(len(act))
        self.alt = alt.astype(np.int32)
        self.n_active = len(act)
        self.elems = np.concatenate(
            [m.elems + offs[i] for i, m in enumerate(self.meshes) if m.isDeformable]
            or [np.zeros((0, 4), np.int64)]).astype(np.int32)
        self.czs = np.concatenate(
            [m.czs + offs[i] for i, m in enumerate(self.meshes) if m.isDeformable]
            or [np.zeros((0, 6), np.int64)]).astype(np.int32).reshape(-1, 6)
        self.faces = np.concatenate([m.faces + offs[i] for i, m in enumerate(self.meshes)]).astype(np.int32)
        # surface elements and their adjacent faces (Mesh.cs:665-678, Element.cs:15-20)
        sel, smesh, adj_lists = [], [], []
        for i, m in enumerate(self.meshes):
            on_face = np.zeros(m.n_nodes, bool)
            on_face[m.faces.ravel()] = True
            s = np.nonzero(on_face[m.elems].any(axis=1))[0]
            sel.append(m.elems[s] + offs[i])
            smesh.append(np.full(len(s), i))
            adj_lists.append(_adjacent_faces(m.elems[s], m.faces, m.n_nodes) )
        self.selem = np.concatenate(sel).astype(np.int32)
        self.selem_mesh = np.concatenate(smesh)
        off = [0]
        adj = []
        for i, (ao, af) in enumerate(adj_lists):
            adj.append(af + foffs[i])
            off.extend((ao[1:] + off[-1]).tolist())
        self.adj_off = np.asarray(off, np.int32)
        self.adj = (np.concatenate(adj) if adj else np.zeros(0)).astype(np.int32)
        return self


def _adjacent_faces(el: np.ndarray, faces: np.ndarray, n_nodes: int):
    """Ordered unique faces touching any vertex of each element, in the order
    vertex 0..3 then each vertex's faces in face order (Element.FindAdjFaces)."""
    fv = faces.ravel()
    fid = np.repeat(np.arange(len(faces)), 3)
    o = np.lexsort((fid, fv))
    fv, fid = fv[o], fid[o]
    noff = np.searchsorted(fv, np.arange(n_nodes + 1))
    cnt = noff[1:] - noff[:-1]
    ne = len(el)
    c = cnt[el]                                   # [ne, 4]
    tot = c.sum(axis=1)
    e_rep = np.repeat(np.arange(ne), tot)
    v_rep = np.repeat(el.ravel(), c.ravel())
    vi_rep = np.repeat(np.tile(np.arange(4), ne), c.ravel())
    start = np.repeat(noff[el.ravel()], c.ravel())
    within = np.arange(len(v_rep)) - np.repeat(np.cumsum(c.ravel()) - c.ravel(), c.ravel())
    f_rep = fid[start + within]
    rank = vi_rep * (1 << 20) + within
    # first occurrence of each (element, face)
    o = np.lexsort((rank, f_rep, e_rep))
    e_s, f_s, r_s = e_rep[o], f_rep[o], rank[o]
    first = np.ones(len(e_s), bool)
    first[1:] = (e_s[1:] != e_s[:-1]) | (f_s[1:] != f_s[:-1])
    e_s, f_s, r_s = e_s[first], f_s[first], r_s[first]
    o = np.lexsort((r_s, e_s))
    e_s, f_s = e_s[o], f_s[o]
    off = np.searchsorted(e_s, np.arange(ne + 1))
    return off.astype(np.int64), f_s.astype(np.int64)


def candidate_pairs(coll: Collection, xt: np.ndarray, pad: float = 0.0,
                    max_pairs: int | None = None, same_mesh: bool = True,
                    vertex_in_box: bool = True) -> np.ndarray:
    """Surface-element pairs whose bounding boxes overlap, that share no node
    and where a vertex of one lies in the other's box; with same_mesh=False
    only pairs of different meshes.

    Host stand-in for the reference's k-DOP broad phase (v3Library/Collisions/
    BVH), whose tree holds every surface element of every mesh: pairs of one
    mesh are candidates too, and across a grain boundary (split nodes) they
    give impacts.  Pairs are also dropped unless a vertex of one element lies
    in the other's box, which every impact needs.  A k-DOP contains the box's
    slabs, so these pairs include every k-DOP pair that can give an impact.
    Returns [n, 2] int32 surface-element ids, ascending."""
    se = coll.selem
    lo = xt[se].min(axis=1) - pad
    hi = xt[se].max(axis=1) + pad
    cell = float(np.max(hi - lo)) if len(se) else 1.0
    base = lo.min(axis=0)
    clo = np.floor((lo - base) / cell).astype(np.int64)
    chi = np.floor((hi - base) / cell).astype(np.int64)
    ent_e, ent_c = [], []
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                c = clo + np.array([dx, dy, dz])
                ok = np.all(c <= chi, axis=1)
                ent_e.append(np.nonzero(ok)[0])
                ent_c.append(c[ok])
    e = np.concatenate(ent_e)
    c = np.concatenate(ent_c)
    key = (c[:, 0] * 1_000_003 + c[:, 1]) * 1_000_033 + c[:, 2]
    o = np.argsort(key, kind="stable")
    key, e = key[o], e[o]
    bounds = np.nonzero(np.r_[True, key[1:] != key[:-1], True])[0]
    out = []
    mesh_of = coll.selem_mesh
    for s, t in zip(bounds[:-1], bounds[1:]):
        m = e[s:t]
        if len(m) < 2:
            continue
        a, b = np.meshgrid(m, m, indexing="ij")
        a, b = a.ravel(), b.ravel()
        k = a < b
        if not same_mesh:
            k &= mesh_of[a] != mesh_of[b]
        a, b = a[k], b[k]
        ov = np.all((lo[a] <= hi[b]) & (lo[b] <= hi[a]), axis=1)
        a, b = a[ov], b[ov]
        ov = ~(se[a][:, :, None] == se[b][:, None, :]).any(axis=(1, 2))
        if vertex_in_box:
            # a vertex of one inside the other's box: an impact needs a vertex
            # inside the other tet
            a, b = a[ov], b[ov]
            va, vb = xt[se[a]], xt[se[b]]
            ov = (np.all((va >= lo[b][:, None]) & (va <= hi[b][:, None]), axis=2).any(axis=1) |
                  np.all((vb >= lo[a][:, None]) & (vb <= hi[a][:, None]), axis=2).any(axis=1))
        if ov.any():
            out.append(np.stack([a[ov], b[ov]], 1))
    if not out:
        return np.zeros((0, 2), np.int32)
    p = np.unique(np.concatenate(out), axis=0)
    if max_pairs is not None:
        p = p[:max_pairs]
    return p.astype(np.int32)


# ---- the benchmark configurations --------------------------------------------------

def cantilever(seed: int = 0) -> Collection:
    """Beam 0.6 x 0.1 x 0.1 m, 24 x 4 x 4 hexahedra (2304 tets), two grains
    split at x = 0.3 (32 CZs), root face anchored, tip face displaced."""
    m = box_mesh((24, 4, 4), (0.6, 0.1, 0.1), name="beam")
    g = (m.x0[m.elems].mean(axis=1)[:, 0] > 0.3).astype(np.int64)
    m = insert_czs(m, g)
    root = np.isclose(m.x0[:, 0], 0.0)
    tip = np.isclose(m.x0[:, 0], 0.6)
    m.anchored = root | tip
    m.forced = [(tip, 0.0, 0.0, 1e-3, 1.0)]  # 1 mm/s along z
    return Collection([m]).prepare()


def polycrystal(n: int = 32, grains: int = 128, edge: float = 1e-3, seed: int = 0,
                platens: bool = True, gap: float = -0.25, platen_cells: int | None = None) -> Collection:
    """Cube of n^3 hexahedra (6 n^3 tets) with `grains` Voronoi grains and CZs on
    every grain boundary, between two rigid platens.  `gap` is the platen
    clearance in cell sizes (negative: the platens already overlap the cube)."""
    h = edge / n
    m = box_mesh((n, n, n), (edge, edge, edge), name="cube")
    g = voronoi_grains(m.x0, m.elems, grains, seed, lo=(0, 0, 0), hi=(edge, edge, edge))
    m = insert_czs(m, g)
    meshes = [m]
    if platens:
        pc = platen_cells or max(2, n // 4)
        ext = edge * 1.25
        o = -0.125 * edge
        th = 2 * h
        top = box_mesh((pc, pc, 1), (ext, ext, th), (o, o, edge + gap * h), deformable=False, name="top")
        bot = box_mesh((pc, pc, 1), (ext, ext, th), (o, o, -th - gap * h), deformable=False, name="bottom")
        top.velocity = (0.0, 0.0, -0.05)
        bot.velocity = (0.0, 0.0, 0.05)
        meshes += [top, bot]
    return Collection(meshes).prepare()


def ice_impact(n: int = 40, grains: int = 64, seed: int = 0, size=(0.2, 0.2, 0.1), gap: float = 1e-4,
               speed: float = 2.5, shift=(0.37, 0.21)):
    """Two ice blocks colliding: each size[0] x size[1] x size[2] m, n x n x
    n/2 hexahedra (3 n^3 tets; n = 40 gives 192,000 tets per block), `grains`
    Voronoi grains with CZs on every grain boundary; block B sits `gap` m above
    block A, shifted in x and y by `shift` times the hexahedron edge, and they
    approach at +-speed m/s along z (5 m/s relative by default: the 0.1 mm gap
    closes in 4 steps of 5 us).  Without the shift both blocks share one x-y
    grid, every node of A's top face meets a vertical edge of B's bottom layer,
    and the point-in-tet test (strict inequalities) contains it in no tet.  No
    node is anchored.
    Returns the collection and the initial velocity of every node [N, 3] (the
    reference has no such input, ImplicitModel3 starts at rest; v0 is
    ImplicitModel3's extension for this workload)."""
    nz = max(1, n // 2)
    meshes = []
    for k, (z0, name) in enumerate(((0.0, "blockA"), (size[2] + gap, "blockB"))):
        ox = k * shift[0] * size[0] / n
        oy = k * shift[1] * size[1] / n
        m = box_mesh((n, n, nz), size, (ox, oy, z0), name=name)
        g = voronoi_grains(m.x0, m.elems, grains, seed * 1000 + k, lo=(ox, oy, z0),
                           hi=(ox + size[0], oy + size[1], z0 + size[2]))
        meshes.append(insert_czs(m, g))
    coll = Collection(meshes).prepare()
    v0 = np.zeros_like(coll.x0)
    na = meshes[0].n_nodes
    v0[:na, 2] = speed
    v0[na:, 2] = -speed
    return coll, v0


def batched_specimens(n_specimens: int = 64, seed: int = 0, tets=(5000, 60000), grains=(8, 64),
                      edge: float = 1e-3, spacing: float = 0.0, only: list | None = None):
    """Independent polycrystal cubes of uneven size: specimen i has about
    U[tets] tetrahedra (a cube of n^3 hexahedra, n = round((t / 6)^(1/3))) and
    U[grains] Voronoi grains with CZs on every grain boundary.  Specimen i
    sits at x = i * spacing * edge.  The default 0 keeps every specimen in its
    own frame at the origin: the specimens never interact, and a frame far
    from the origin costs accuracy, because the corotational forces subtract
    rest coordinates from rotated current ones (xr = R^T xc - x0) and lose the
    digits of the offset.  `only` keeps a subset of the specimen indices (the
    draw for every index is the same whether or not it is kept).  Returns the
    collection and, per kept specimen, (index, tets, grains)."""
    rng = np.random.default_rng(seed)
    draws = [(int(rng.integers(tets[0], tets[1] + 1)), int(rng.integers(grains[0], grains[1] + 1)))
             for _ in range(n_specimens)]
    keep = range(n_specimens) if only is None else sorted(only)
    meshes, info = [], []
    for i in keep:
        t, g = draws[i]
        n = max(2, int(round((t / 6.0) ** (1.0 / 3.0))))
        m = box_mesh((n, n, n), (edge, edge, edge), (i * spacing * edge, 0.0, 0.0), name=f"specimen{i}")
        lo = (i * spacing * edge, 0.0, 0.0)
        hi = (i * spacing * edge + edge, edge, edge)
        gr = voronoi_grains(m.x0, m.elems, g, seed * 1000 + i, lo=lo, hi=hi)
        m = insert_czs(m, gr)
        meshes.append(m)
        info.append((i, 6 * n ** 3, g))
    return Collection(meshes).prepare(), info


def lognormal_strengths(n_cz: int, mean: float = 1e6, cv: float = 0.2, seed: int = 0,
                        granule_pairs: np.ndarray | None = None) -> np.ndarray:
    """Per-CZ strength, lognormal with the given mean and coefficient of
    variation, drawn per grain boundary (one value per grain pair)."""
    rng = np.random.default_rng(seed + 7919)
    s2 = np.log(1 + cv * cv)
    mu = np.log(mean) - 0.5 * s2
    if granule_pairs is None:
        return rng.lognormal(mu, np.sqrt(s2), n_cz)
    _, inv = np.unique(granule_pairs, axis=0, return_inverse=True)
    vals = rng.lognormal(mu, np.sqrt(s2), inv.max() + 1)
    return vals[inv.ravel()]
