"""icFlow's snapshot files: one mesh frame (`.mg`) and one saved step (`.mgs`).

A frame (Mesh.SaveFrame / LoadFrame, v3Library/Geometry/Mesh/Mesh.cs:106-384)
is written with .NET's BinaryWriter (little endian, a bool in one byte, a
string as a 7-bit length then UTF-8):

  bool isDeformable, isIndenter, isFloor, hide; string name
  int32 nNodes, nElems, nCZs, nFaces, nEdges
  int32[iSize]   per element: 4 node ids, grain              (eli_str = 5)
                 per CZ: 6 node ids, 2 face ids, immutable id (czi_str = 9)
                 per face: 3 node ids, grain, element or -1  (fi_str = 5)
                 per grain edge: 2 node ids                  (gei_str = 2)
  bool[bSize]    per CZ: failed; per face: exposed, created; per edge: exposed
  double[dSize]  per node: x0 y0 z0, ux uy uz, vx vy vz, ax ay az (ndd_str = 12)
                 per CZ: pmax[3], tmax[3], avgDn, avgDt, avgTn, avgTt,
                 maxAvgDn, maxAvgDt                           (czd_str = 12)
  BinaryFormatter: List<SurfaceFragment>, then TranslationCollection

A step snapshot (ImplicitModel3.SaveStep, ImplicitModel3.cs:444-462, through
MeshCollection.Save and WriteImpacts, MeshCollection.cs:113-118,163-175) is
int32 nMeshes, each mesh's frame, then int32 nCollisions, int32 stride and,
when there are impacts, int32[4 stride] in the strided layout
collisions[i + k stride] (node, then the face's three nodes).

The BinaryFormatter objects are read and written through `nrbf`.  The frame
part is exact; the two .NET objects follow the published stream grammar and
the class layout of SurfaceFragment.cs and Translation.cs (field order as
declared, auto properties as "<name>k__BackingField"), unverified against a
.NET runtime (none here).
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

from icflow_b200 import nrbf

LIBRARY = "icFlowLibrary, Version=3.0.0.0, Culture=neutral, PublicKeyToken=null"
_FRAG = "icFlow.SurfaceFragment"
_ROLE = "icFlow.SurfaceFragment+SurfaceRole"
_TRANS = "icFlow.Translation"
_TCOLL = "icFlow.TranslationCollection"
_LIST_FRAG = f"System.Collections.Generic.List`1[[{_FRAG}, {LIBRARY}]]"
_LIST_INT = f"System.Collections.Generic.List`1[[System.Int32, {nrbf.MSCORLIB}]]"
# SurfaceFragment's serialized fields in declaration order (allFaces and
# _nodes are [NonSerialized]); the doubles after role
_FRAG_DOUBLES = ("px", "py", "pz", "dx", "dy", "dz", "fx", "fy", "fz", "area", "applicationTime")


def _bf(name):
    return f"<{name}>k__BackingField"


@dataclass
class SurfaceFragment:
    """SurfaceFragment.cs: a set of faces with a role (0 Free, 1 Anchored,
    2 Forced) and its prescribed stress/displacement."""
    id: int = 0
    sensor: bool = False
    faces: list = field(default_factory=list)
    role: int = 0
    px: float = 0.0
    py: float = 0.0
    pz: float = 0.0
    dx: float = 0.0
    dy: float = 0.0
    dz: float = 0.0
    fx: float = 0.0
    fy: float = 0.0
    fz: float = 0.0
    area: float = 0.0
    applicationTime: float = 1000.0


@dataclass
class Translation:
    """Translation.cs: a rigid offset (dx, dy, dz) reached at time t."""
    dx: float = 0.0
    dy: float = 0.0
    dz: float = 0.0
    t: float = 0.0


@dataclass
class MeshFrame:
    """Everything a frame file holds for one mesh."""
    name: str = ""
    isDeformable: bool = True
    isIndenter: bool = False
    isFloor: bool = False
    hide: bool = False
    x0: np.ndarray = None            # [n, 3]
    u: np.ndarray = None             # [n, 3]
    v: np.ndarray = None             # [n, 3]
    a: np.ndarray = None             # [n, 3]
    elems: np.ndarray = None         # [ne, 4] int32
    elem_granule: np.ndarray = None  # [ne]
    czs: np.ndarray = None           # [nc, 6]
    cz_faces: np.ndarray = None      # [nc, 2]
    cz_immutable: np.ndarray = None  # [nc]
    cz_pmax: np.ndarray = None       # [nc, 3]
    cz_tmax: np.ndarray = None       # [nc, 3]
    cz_avg: np.ndarray = None        # [nc, 4] avgDn, avgDt, avgTn, avgTt
    cz_maxavg: np.ndarray = None     # [nc, 2] maxAvgDn, maxAvgDt
    cz_failed: np.ndarray = None     # [nc] bool
    faces: np.ndarray = None         # [nf, 3]
    face_granule: np.ndarray = None  # [nf]
    face_elem: np.ndarray = None     # [nf], -1 none
    face_exposed: np.ndarray = None  # [nf] bool
    face_created: np.ndarray = None  # [nf] bool
    edges: np.ndarray = None         # [ned, 2]
    edge_exposed: np.ndarray = None  # [ned] bool
    surface_fragments: list = field(default_factory=list)
    translations: list = field(default_factory=list)


# ---- BinaryWriter primitives ---------------------------------------------------
def _w_str(out, s: str):
    data = s.encode("utf-8")
    n = len(data)
    while True:
        c = n & 0x7F
        n >>= 7
        out.write(bytes([c | (0x80 if n else 0)]))
        if not n:
            break
    out.write(data)


def _r_str(buf, pos):
    n, shift = 0, 0
    while True:
        c = buf[pos]
        pos += 1
        n |= (c & 0x7F) << shift
        shift += 7
        if not c & 0x80:
            break
    return buf[pos:pos + n].decode("utf-8"), pos + n


def _z(shape, dtype):
    return np.zeros(shape, dtype)


def _complete(f: MeshFrame) -> MeshFrame:
    """Zero-filled defaults for the parts a caller left out."""
    n = len(f.x0)
    for k in ("u", "v", "a"):
        if getattr(f, k) is None:
            setattr(f, k, _z((n, 3), np.float64))
    ne = 0 if f.elems is None else len(f.elems)
    if f.elems is None:
        f.elems = _z((0, 4), np.int32)
    if f.elem_granule is None:
        f.elem_granule = _z(ne, np.int32)
    nc = 0 if f.czs is None else len(f.czs)
    defaults = {"czs": ((nc, 6), np.int32), "cz_faces": ((nc, 2), np.int32),
                "cz_pmax": ((nc, 3), np.float64), "cz_tmax": ((nc, 3), np.float64), "cz_avg": ((nc, 4), np.float64),
                "cz_maxavg": ((nc, 2), np.float64), "cz_failed": (nc, bool)}
    for k, (sh, dt) in defaults.items():
        if getattr(f, k) is None:
            setattr(f, k, _z(sh, dt))
    if f.cz_immutable is None:  # CZ.immutableID: the CZ's index when it was created
        f.cz_immutable = np.arange(nc, dtype=np.int32)
    nf = 0 if f.faces is None else len(f.faces)
    if f.faces is None:
        f.faces = _z((0, 3), np.int32)
    for k, dt, fill in (("face_granule", np.int32, 0), ("face_elem", np.int32, -1), ("face_exposed", bool, True),
                        ("face_created", bool, False)):
        if getattr(f, k) is None:
            setattr(f, k, np.full(nf, fill, dt))
    if f.edges is None:
        f.edges = _z((0, 2), np.int32)
    if f.edge_exposed is None:
        f.edge_exposed = _z(len(f.edges), bool)
    return f


# ---- the two BinaryFormatter objects ---------------------------------------------
def _fragments_blob(frags) -> bytes:
    """List<SurfaceFragment> as BinaryFormatter lays it out: the list, its
    _items array (capacity a power of two), each fragment with its faces
    list (List<int>: _items, _size, _version) and its role (an enum boxed
    inline with member value__)."""
    w = nrbf.Writer(LIBRARY)
    w.begin(1)
    root = w.new_id()
    w.lib()
    items = w.new_id()
    cap = 0 if not frags else max(4, 1 << (len(frags) - 1).bit_length())
    w.class_record(root, _LIST_FRAG, [("_items", nrbf.BT_CLASS, _FRAG + "[]", items),
                                      ("_size", nrbf.BT_PRIMITIVE, nrbf.P_INT32, len(frags)),
                                      ("_version", nrbf.BT_PRIMITIVE, nrbf.P_INT32, len(frags))], system=True)
    ids = [w.new_id() for _ in frags]
    w.class_array(items, _FRAG, ids, cap)
    lists = []
    for oid, fr in zip(ids, frags):
        lid = w.new_id()
        lists.append((lid, fr))
        role = int(fr.role)

        def enum_value(role=role):
            w.class_record(w.new_id(), _ROLE, [("value__", nrbf.BT_PRIMITIVE, nrbf.P_INT32, role)])

        members = [(_bf("id"), nrbf.BT_PRIMITIVE, nrbf.P_INT32, int(fr.id)),
                   (_bf("sensor"), nrbf.BT_PRIMITIVE, nrbf.P_BOOLEAN, bool(fr.sensor)),
                   ("faces", nrbf.BT_SYSTEM_CLASS, _LIST_INT, lid),
                   (_bf("role"), nrbf.BT_CLASS, _ROLE, enum_value)]
        members += [(_bf(k), nrbf.BT_PRIMITIVE, nrbf.P_DOUBLE, float(getattr(fr, k))) for k in _FRAG_DOUBLES]
        w.class_record(oid, _FRAG, members)
    for lid, fr in lists:
        arr = w.new_id()
        faces = [int(x) for x in fr.faces]
        cap = 0 if not faces else max(4, 1 << (len(faces) - 1).bit_length())
        w.class_record(lid, _LIST_INT, [("_items", nrbf.BT_PRIMITIVE_ARRAY, nrbf.P_INT32, arr),
                                        ("_size", nrbf.BT_PRIMITIVE, nrbf.P_INT32, len(faces)),
                                        ("_version", nrbf.BT_PRIMITIVE, nrbf.P_INT32, len(faces))], system=True)
        w.primitive_array(arr, nrbf.P_INT32, faces + [0] * (cap - len(faces)))
    return w.end()


def _translations_blob(trans) -> bytes:
    """TranslationCollection (a List<Translation>): its inherited fields under
    the base class's name, then each Translation's four doubles."""
    w = nrbf.Writer(LIBRARY)
    w.begin(1)
    root = w.new_id()
    w.lib()
    items = w.new_id()
    cap = 0 if not trans else max(4, 1 << (len(trans) - 1).bit_length())
    w.class_record(root, _TCOLL, [("List`1+_items", nrbf.BT_CLASS, _TRANS + "[]", items),
                                  ("List`1+_size", nrbf.BT_PRIMITIVE, nrbf.P_INT32, len(trans)),
                                  ("List`1+_version", nrbf.BT_PRIMITIVE, nrbf.P_INT32, len(trans))])
    ids = [w.new_id() for _ in trans]
    w.class_array(items, _TRANS, ids, cap)
    for oid, t in zip(ids, trans):
        w.class_record(oid, _TRANS, [(_bf(k), nrbf.BT_PRIMITIVE, nrbf.P_DOUBLE, float(getattr(t, k)))
                                     for k in ("dx", "dy", "dz", "t")])
    return w.end()


def _fragments_from(obj) -> list:
    out = []
    for o in nrbf.list_items(obj):
        if o is None:
            continue
        fr = SurfaceFragment()
        fr.id = int(o.member(_bf("id")))
        fr.sensor = bool(o.member(_bf("sensor")))
        fr.faces = [int(x) for x in nrbf.list_items(o.member("faces"))]
        role = o.member(_bf("role"))
        fr.role = int(role.member("value__")) if isinstance(role, nrbf.NrbfObject) else int(role)
        for k in _FRAG_DOUBLES:
            setattr(fr, k, float(o.member(_bf(k))))
        out.append(fr)
    return out


def _translations_from(obj) -> list:
    out = []
    for o in nrbf.list_items(obj):
        if o is None:
            continue
        out.append(Translation(*(float(o.member(_bf(k))) for k in ("dx", "dy", "dz", "t"))))
    return out


# ---- frames -----------------------------------------------------------------------
def write_frame(out, f: MeshFrame) -> None:
    """Mesh.SaveFrame (Mesh.cs:106-261) to a binary stream."""
    f = _complete(f)
    nn, ne, nc, nf, ned = len(f.x0), len(f.elems), len(f.czs), len(f.faces), len(f.edges)
    for b in (f.isDeformable, f.isIndenter, f.isFloor, f.hide):
        out.write(struct.pack("<?", bool(b)))
    _w_str(out, f.name)
    out.write(struct.pack("<5i", nn, ne, nc, nf, ned))
    isn = np.concatenate([
        np.concatenate([f.elems.reshape(ne, 4), f.elem_granule.reshape(ne, 1)], 1).ravel(),
        np.concatenate([f.czs.reshape(nc, 6), f.cz_faces.reshape(nc, 2), f.cz_immutable.reshape(nc, 1)], 1).ravel(),
        np.concatenate([f.faces.reshape(nf, 3), f.face_granule.reshape(nf, 1), f.face_elem.reshape(nf, 1)], 1).ravel(),
        f.edges.reshape(ned, 2).ravel()]).astype("<i4")
    bsn = np.concatenate([f.cz_failed.ravel(),
                          np.stack([f.face_exposed, f.face_created], 1).ravel() if nf else np.zeros(0, bool),
                          f.edge_exposed.ravel()]).astype(np.uint8)
    dsn = np.concatenate([
        np.concatenate([f.x0, f.u, f.v, f.a], 1).ravel(),
        np.concatenate([f.cz_pmax.reshape(nc, 3), f.cz_tmax.reshape(nc, 3), f.cz_avg.reshape(nc, 4),
                        f.cz_maxavg.reshape(nc, 2)], 1).ravel()]).astype("<f8")
    out.write(isn.tobytes())
    out.write(bsn.tobytes())
    out.write(dsn.tobytes())
    out.write(_fragments_blob(f.surface_fragments))
    out.write(_translations_blob(f.translations))


def read_frame(buf: bytes, pos: int = 0):
    """Mesh.LoadFrame (Mesh.cs:262-384) from bytes at `pos`; returns
    (MeshFrame, end position).  Raises ValueError on a truncated or
    malformed frame."""
    try:
        f = MeshFrame()
        f.isDeformable, f.isIndenter, f.isFloor, f.hide = struct.unpack_from("<4?", buf, pos)
        f.name, pos = _r_str(buf, pos + 4)
        nn, ne, nc, nf, ned = struct.unpack_from("<5i", buf, pos)
        pos += 20
    except (struct.error, IndexError, UnicodeDecodeError) as e:
        raise ValueError(f"frame header: {e}") from e
    if min(nn, ne, nc, nf, ned) < 0:
        raise ValueError("negative count in frame header")
    i_size = 5 * ne + 9 * nc + 5 * nf + 2 * ned
    b_size = 2 * nf + ned + nc
    d_size = 12 * nn + 12 * nc
    need = 4 * i_size + b_size + 8 * d_size
    if pos + need > len(buf):
        raise ValueError("frame ends inside its arrays")
    isn = np.frombuffer(buf, "<i4", i_size, pos).astype(np.int32)
    pos += 4 * i_size
    bsn = np.frombuffer(buf, np.uint8, b_size, pos).astype(bool)
    pos += b_size
    dsn = np.frombuffer(buf, "<f8", d_size, pos).astype(np.float64)
    pos += 8 * d_size
    o = 0
    e = isn[o:o + 5 * ne].reshape(ne, 5)
    o += 5 * ne
    f.elems, f.elem_granule = e[:, :4].copy(), e[:, 4].copy()
    c = isn[o:o + 9 * nc].reshape(nc, 9)
    o += 9 * nc
    f.czs, f.cz_faces, f.cz_immutable = c[:, :6].copy(), c[:, 6:8].copy(), c[:, 8].copy()
    fc = isn[o:o + 5 * nf].reshape(nf, 5)
    o += 5 * nf
    f.faces, f.face_granule, f.face_elem = fc[:, :3].copy(), fc[:, 3].copy(), fc[:, 4].copy()
    f.edges = isn[o:o + 2 * ned].reshape(ned, 2).copy()
    f.cz_failed = bsn[:nc].copy()
    fb = bsn[nc:nc + 2 * nf].reshape(nf, 2)
    f.face_exposed, f.face_created = fb[:, 0].copy(), fb[:, 1].copy()
    f.edge_exposed = bsn[nc + 2 * nf:].copy()
    nd = dsn[:12 * nn].reshape(nn, 12)
    f.x0, f.u, f.v, f.a = nd[:, 0:3].copy(), nd[:, 3:6].copy(), nd[:, 6:9].copy(), nd[:, 9:12].copy()
    cd = dsn[12 * nn:].reshape(nc, 12)
    f.cz_pmax, f.cz_tmax, f.cz_avg, f.cz_maxavg = cd[:, 0:3].copy(), cd[:, 3:6].copy(), cd[:, 6:10].copy(), cd[:, 10:12].copy()
    for arr, lim, what in ((f.elems, nn, "element node"), (f.czs, nn, "CZ node"), (f.faces, nn, "face node"),
                           (f.edges, nn, "edge node"), (f.cz_faces, nf, "CZ face")):
        if arr.size and (arr.min() < 0 or arr.max() >= lim):
            raise ValueError(f"{what} index out of range")
    if f.face_elem.size and (f.face_elem.min() < -1 or f.face_elem.max() >= ne):
        raise ValueError("face element index out of range")
    frags, pos = nrbf.read(buf, pos)
    trans, pos = nrbf.read(buf, pos)
    f.surface_fragments = _fragments_from(frags)
    f.translations = _translations_from(trans)
    return f, pos


def save_mg(path, f: MeshFrame) -> None:
    with open(path, "wb") as out:
        write_frame(out, f)


def load_mg(path) -> MeshFrame:
    with open(path, "rb") as fh:
        buf = fh.read()
    return read_frame(buf, 0)[0]


# ---- steps --------------------------------------------------------------------------
def write_step(out, frames, impacts=None) -> None:
    """A step snapshot: MeshCollection.Save then WriteImpacts.  `impacts`:
    [n, 4] (node, face nodes), written in the strided layout with stride n."""
    out.write(struct.pack("<i", len(frames)))
    for f in frames:
        write_frame(out, f)
    imp = np.zeros((0, 4), np.int32) if impacts is None else np.asarray(impacts, np.int32).reshape(-1, 4)
    n = len(imp)
    out.write(struct.pack("<2i", n, n))
    if n:
        out.write(np.ascontiguousarray(imp.T).astype("<i4").tobytes())


def read_step(buf: bytes):
    """(frames, impacts [n, 4]) of a step snapshot."""
    if len(buf) < 4:
        raise ValueError("empty step snapshot")
    (nm,) = struct.unpack_from("<i", buf, 0)
    if nm <= 0:
        raise ValueError("step snapshot without meshes")
    pos = 4
    frames = []
    for _ in range(nm):
        f, pos = read_frame(buf, pos)
        frames.append(f)
    if pos + 8 > len(buf):
        raise ValueError("step snapshot ends before its impacts")
    n, stride = struct.unpack_from("<2i", buf, pos)
    pos += 8
    if n < 0 or stride < n:
        raise ValueError("bad impact count")
    if n == 0:
        return frames, np.zeros((0, 4), np.int32)
    if pos + 16 * stride > len(buf):
        raise ValueError("step snapshot ends inside its impacts")
    c = np.frombuffer(buf, "<i4", 4 * stride, pos).reshape(4, stride)
    return frames, np.ascontiguousarray(c[:, :n].T).astype(np.int32)


def save_mgs(path, frames, impacts=None) -> None:
    with open(path, "wb") as out:
        write_step(out, frames, impacts)


def load_mgs(path):
    with open(path, "rb") as fh:
        return read_step(fh.read())


# ---- to and from the package's meshes ----------------------------------------------
def frame_of_mesh(m, u=None, v=None, a=None, pmax=None, tmax=None, failed=None) -> MeshFrame:
    """A MeshFrame of a `mesh.Mesh` (its node state and CZ state optional)."""
    f = MeshFrame(name=m.name, isDeformable=bool(m.isDeformable), x0=np.asarray(m.x0, np.float64),
                  u=None if u is None else np.asarray(u, np.float64),
                  v=None if v is None else np.asarray(v, np.float64),
                  a=None if a is None else np.asarray(a, np.float64),
                  elems=np.asarray(m.elems, np.int32),
                  elem_granule=None if m.granule is None else np.asarray(m.granule, np.int32),
                  czs=np.asarray(m.czs, np.int32), cz_faces=np.asarray(m.cz_faces, np.int32),
                  cz_pmax=None if pmax is None else np.asarray(pmax, np.float64),
                  cz_tmax=None if tmax is None else np.asarray(tmax, np.float64),
                  cz_failed=None if failed is None else np.asarray(failed, bool),
                  faces=np.asarray(m.faces, np.int32), face_exposed=np.asarray(m.face_exposed, bool))
    return _complete(f)


def mesh_of_frame(f: MeshFrame):
    """A `mesh.Mesh` of a frame: geometry, elements, faces, CZs, grains and
    the anchored nodes of its Anchored surface fragments."""
    from icflow_b200 import mesh as M

    m = M.Mesh(x0=f.x0.copy(), elems=f.elems.astype(np.int64), faces=f.faces.astype(np.int64),
               face_exposed=f.face_exposed.copy(), czs=f.czs.astype(np.int64), cz_faces=f.cz_faces.astype(np.int64),
               granule=f.elem_granule.copy(), isDeformable=bool(f.isDeformable), name=f.name)
    anchored = np.zeros(len(f.x0), bool)
    for fr in f.surface_fragments:
        if fr.role == 1 and fr.faces:
            anchored[f.faces[np.asarray(fr.faces)].ravel()] = True
    m.anchored = anchored
    return m
