"""Gmsh 2.2 ASCII meshes in and out (v3Library/Geometry/Mesh/Mesh.cs:548-616).

icFlow reads its polycrystal setups from `.msh` files: a `$Nodes` block of
"id x y z" lines, then an `$Elements` block whose lines are
"id type ntags tag1 .. tagN node1 .. nodeK" with 1-based node numbers.  It keeps
three element types (LoadMsh, Mesh.cs:575-612):

* 4, a linear tetrahedron: an element of the mesh, its grain (`granule`) the
  second tag minus one;
* 2, a triangle: a face of the mesh;
* 1, a line: a grain edge.

Nodes are numbered in the order they appear (the reference ignores the node
ids of the `$Nodes` block and assumes they run 1..n).  The reference's files
carry three tags per element and it reads the nodes from the seventh field;
here the node fields start after `ntags`, which is the same for those files
and also reads files with two or four tags.

`load_msh` turns a file into a `Mesh` of this package: the boundary faces of
the tets become its exposed faces and, when the file has more than one grain,
cohesive zones are inserted on every face between two grains
(`mesh.insert_czs`, CZInsertionTool.cs:371-491).  The six surface fragments
that the reference derives from the triangles for its boundary conditions
(DetectSurfacesAfterLoadingMSH, Mesh.cs:618-663) are left to the caller, who
marks anchored and driven nodes on the returned mesh.
"""
from __future__ import annotations

import io
import os
from dataclasses import dataclass

import numpy as np

from icflow_b200 import mesh as M


@dataclass
class MshData:
    x0: np.ndarray         # [n, 3] node positions, in file order
    elems: np.ndarray      # [ne, 4] tets, 0-based node indices
    granule: np.ndarray    # [ne] grain of every tet (second tag - 1)
    triangles: np.ndarray  # [nt, 3] 0-based
    edges: np.ndarray      # [ned, 2] 0-based


def read_msh(source) -> MshData:
    """Parses a Gmsh 2.2 ASCII mesh from a path, a text stream or a string
    holding the file's contents.  Raises ValueError on a malformed file."""
    if isinstance(source, (str, os.PathLike)) and os.path.exists(source):
        with open(source, "r") as f:
            lines = f.read().splitlines()
    elif isinstance(source, str):
        lines = source.splitlines()
    else:
        lines = source.read().splitlines()
    it = iter(lines)
    for s in it:
        if s.strip() == "$Nodes":
            break
    else:
        raise ValueError("no $Nodes block")
    try:
        n_nodes = int(next(it).split()[0])
    except (StopIteration, ValueError):
        raise ValueError("bad node count") from None
    xs = []
    for s in it:
        s = s.strip()
        if s == "$EndNodes":
            break
        p = s.split()
        if len(p) < 4:
            continue
        xs.append((float(p[1]), float(p[2]), float(p[3])))
    else:
        raise ValueError("no $EndNodes")
    if len(xs) != n_nodes:
        raise ValueError(f"$Nodes announces {n_nodes} nodes, the block has {len(xs)}")
    for s in it:
        if s.strip() == "$Elements":
            break
        if s.strip():
            raise ValueError("no $Elements tag after $EndNodes")
    else:
        raise ValueError("no $Elements block")
    next(it, None)  # element count (the reference does not check it either)
    tets, gran, tris, eds = [], [], [], []
    for s in it:
        s = s.strip()
        if s == "$EndElements":
            break
        p = s.split()
        if len(p) < 3:
            continue
        typ, ntags = int(p[1]), int(p[2])
        nodes = [int(v) - 1 for v in p[3 + ntags:]]
        if typ == 4:
            if ntags < 2 or len(nodes) < 4:
                raise ValueError(f"tetrahedron line without a grain tag or four nodes: {s!r}")
            tets.append(nodes[:4])
            gran.append(int(p[4]) - 1)
        elif typ == 2:
            tris.append(nodes[:3])
        elif typ == 1:
            eds.append(nodes[:2])
    else:
        raise ValueError("no $EndElements")
    el = np.asarray(tets, np.int64).reshape(-1, 4)
    if el.size and (el.min() < 0 or el.max() >= n_nodes):
        raise ValueError("a tetrahedron references a node outside the $Nodes block")
    return MshData(x0=np.asarray(xs, np.float64).reshape(-1, 3), elems=el,
                   granule=np.asarray(gran, np.int64),
                   triangles=np.asarray(tris, np.int64).reshape(-1, 3),
                   edges=np.asarray(eds, np.int64).reshape(-1, 2))


def write_msh(target, x0: np.ndarray, elems: np.ndarray, granule: np.ndarray | None = None,
              triangles: np.ndarray | None = None) -> None:
    """Writes a Gmsh 2.2 ASCII mesh that `read_msh` and the reference's
    LoadMsh read back: tets with three tags (physical 0, grain + 1, partition
    0), then the triangles, if given.  `target` is a path or a text stream."""
    x0 = np.asarray(x0, np.float64)
    el = np.asarray(elems, np.int64)
    g = np.zeros(len(el), np.int64) if granule is None else np.asarray(granule, np.int64)
    tri = np.zeros((0, 3), np.int64) if triangles is None else np.asarray(triangles, np.int64)
    out = io.StringIO()
    out.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n")
    out.write(f"{len(x0)}\n")
    for i, (x, y, z) in enumerate(x0.tolist()):  # repr of a float reads back exactly
        out.write(f"{i + 1} {x!r} {y!r} {z!r}\n")
    out.write("$EndNodes\n$Elements\n")
    out.write(f"{len(tri) + len(el)}\n")
    k = 1
    for t in tri.tolist():
        out.write(f"{k} 2 3 0 1 0 {t[0] + 1} {t[1] + 1} {t[2] + 1}\n")
        k += 1
    for e, gg in zip(el.tolist(), g.tolist()):
        out.write(f"{k} 4 3 0 {gg + 1} 0 {e[0] + 1} {e[1] + 1} {e[2] + 1} {e[3] + 1}\n")
        k += 1
    out.write("$EndElements\n")
    if isinstance(target, (str, os.PathLike)):
        with open(target, "w") as f:
            f.write(out.getvalue())
    else:
        target.write(out.getvalue())


def load_msh(source, name: str = "", deformable: bool = True, insert_czs: bool = True) -> M.Mesh:
    """A `Mesh` from a Gmsh 2.2 file: its tets, their boundary faces as the
    exposed faces and, with more than one grain and `insert_czs`, cohesive
    zones on every grain boundary (node splitting, one copy per grain)."""
    d = read_msh(source)
    if len(d.elems) == 0:
        raise ValueError("the file has no tetrahedra")
    tf = M._tet_faces(d.elems).reshape(-1, 3)
    keys = M._face_keys(tf)
    _, inv, cnt = np.unique(keys, return_inverse=True, return_counts=True)
    faces = tf[cnt[inv] == 1]
    m = M.Mesh(x0=d.x0, elems=d.elems, faces=faces, face_exposed=np.ones(len(faces), bool),
               isDeformable=deformable, name=name, granule=d.granule)
    if insert_czs and len(np.unique(d.granule)) > 1:
        m = M.insert_czs(m, d.granule)
        m.isDeformable, m.name = deformable, name
    return m
