"""icFlow frame (.mg) and step (.mgs) snapshots (Mesh.cs:106-384,
MeshCollection.cs:113-175, ImplicitModel3.cs:444-462): the binary layout,
round trips of meshes with cohesive zones and their state, surface fragments
and translations, and the .NET serialization records of those two objects."""
import io
import struct

import numpy as np
import pytest

from icflow_b200 import mesh as M
from icflow_b200 import nrbf
from icflow_b200 import snapshot as S


def _frame(seed=0):
    m = M.insert_czs(M.box_mesh((3, 2, 2), (3e-3, 2e-3, 2e-3)), np.repeat(np.arange(2), 36))
    rng = np.random.default_rng(seed)
    n, nc = len(m.x0), len(m.czs)
    f = S.frame_of_mesh(m, u=rng.normal(size=(n, 3)), v=rng.normal(size=(n, 3)), a=rng.normal(size=(n, 3)),
                        pmax=rng.random((nc, 3)), tmax=rng.random((nc, 3)), failed=rng.random(nc) < 0.3)
    f.cz_avg = rng.normal(size=(nc, 4))
    f.cz_maxavg = rng.normal(size=(nc, 2))
    f.face_granule = rng.integers(0, 2, len(f.faces)).astype(np.int32)
    f.face_elem = rng.integers(-1, len(f.elems), len(f.faces)).astype(np.int32)
    f.face_created = rng.random(len(f.faces)) < 0.5
    f.edges = rng.integers(0, n, (5, 2)).astype(np.int32)
    f.edge_exposed = np.array([1, 0, 1, 1, 0], bool)
    f.isIndenter, f.hide = True, True
    f.surface_fragments = [S.SurfaceFragment(id=0, faces=[0, 2, 5], role=1),
                           S.SurfaceFragment(id=1, sensor=True, faces=list(range(7)), role=2, dz=-1e-3,
                                             applicationTime=0.5, area=4e-6),
                           S.SurfaceFragment(id=2)]
    f.translations = [S.Translation(0.0, 0.0, 0.0, 0.0), S.Translation(1e-3, -2e-3, 0.5, 1.5)]
    return m, f


def _same(a: S.MeshFrame, b: S.MeshFrame):
    for k in ("x0", "u", "v", "a", "elems", "elem_granule", "czs", "cz_faces", "cz_immutable", "cz_pmax", "cz_tmax",
              "cz_avg", "cz_maxavg", "cz_failed", "faces", "face_granule", "face_elem", "face_exposed",
              "face_created", "edges", "edge_exposed"):
        assert np.array_equal(np.asarray(getattr(a, k)), np.asarray(getattr(b, k))), k
    for k in ("name", "isDeformable", "isIndenter", "isFloor", "hide"):
        assert getattr(a, k) == getattr(b, k), k
    assert a.surface_fragments == b.surface_fragments
    assert a.translations == b.translations


def test_frame_round_trip():
    _, f = _frame()
    f.name = "grains Ω"
    out = io.BytesIO()
    S.write_frame(out, f)
    g, end = S.read_frame(out.getvalue())
    assert end == len(out.getvalue())
    _same(f, g)


def test_frame_binary_layout():
    """The BinaryWriter part byte for byte: flags, the 7-bit string, counts,
    then the int, bool and double arrays in Mesh.SaveFrame's order."""
    f = S.MeshFrame(name="t", isDeformable=True, isFloor=True,
                    x0=np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float),
                    elems=np.array([[0, 1, 2, 3]], np.int32), elem_granule=np.array([7], np.int32),
                    faces=np.array([[0, 1, 2]], np.int32), face_elem=np.array([0], np.int32))
    f.u = np.arange(12, dtype=float).reshape(4, 3)
    out = io.BytesIO()
    S.write_frame(out, f)
    b = out.getvalue()
    assert b[:4] == bytes([1, 0, 1, 0]) and b[4:6] == b"\x01t"
    assert struct.unpack_from("<5i", b, 6) == (4, 1, 0, 1, 0)
    p = 26
    assert struct.unpack_from("<5i", b, p) == (0, 1, 2, 3, 7)             # element: nodes, grain
    assert struct.unpack_from("<5i", b, p + 20) == (0, 1, 2, 0, 0)        # face: nodes, grain, element
    p += 40
    assert b[p:p + 2] == bytes([1, 0])                                   # face exposed, created
    p += 2
    d = struct.unpack_from("<48d", b, p)
    assert d[:12] == (0, 0, 0, 0, 1, 2, 0, 0, 0, 0, 0, 0)                # node 0: x0, u, v, a
    assert d[12:15] == (1, 0, 0) and d[15:18] == (3, 4, 5)
    assert b[p + 384] == nrbf.HEADER                                     # the .NET objects follow


def test_step_round_trip_with_impacts():
    m, f = _frame(1)
    platen = S.frame_of_mesh(M.box_mesh((2, 2, 1), (3e-3, 3e-3, 1e-3), origin=(0, 0, 2e-3), deformable=False))
    platen.translations = [S.Translation(0, 0, -1e-3, 0.01)]
    imps = np.array([[3, 40, 41, 42], [5, 43, 44, 45], [7, 40, 42, 44]], np.int32)
    out = io.BytesIO()
    S.write_step(out, [f, platen], imps)
    b = out.getvalue()
    frames, got = S.read_step(b)
    assert len(frames) == 2
    _same(f, frames[0])
    _same(platen, frames[1])
    assert np.array_equal(got, imps)
    # WriteImpacts' strided layout: count, stride, then collisions[i + k stride]
    n, stride = struct.unpack_from("<2i", b, len(b) - 8 - 48)
    assert (n, stride) == (3, 3)
    assert struct.unpack_from("<12i", b, len(b) - 48) == tuple(imps.T.ravel())


def test_mesh_of_frame_marks_anchored_fragments():
    m, f = _frame(2)
    g = S.mesh_of_frame(f)
    assert np.array_equal(g.elems, m.elems) and np.array_equal(g.czs, m.czs)
    want = np.zeros(len(m.x0), bool)
    want[f.faces[[0, 2, 5]].ravel()] = True
    assert np.array_equal(g.anchored, want)


def test_truncated_and_corrupt_frames_raise():
    _, f = _frame(3)
    out = io.BytesIO()
    S.write_frame(out, f)
    b = out.getvalue()
    for cut in (3, 20, 40, len(b) // 2, len(b) - 1):
        with pytest.raises(ValueError):
            S.read_frame(b[:cut])
    bad = bytearray(b)
    first_elem = 4 + 1 + len(f.name.encode()) + 20  # flags, name, counts
    assert struct.unpack_from("<i", b, first_elem)[0] == f.elems[0, 0]
    struct.pack_into("<i", bad, first_elem, 10 ** 6)  # element node id out of range
    with pytest.raises(ValueError):
        S.read_frame(bytes(bad))


def _lps(s):
    d = s.encode()
    assert len(d) < 128
    return bytes([len(d)]) + d


def test_nrbf_reader_on_a_hand_built_stream():
    """A stream assembled from the record grammar alone: header; a library; a
    class with a primitive, a string, a reference and a null member; the
    referenced int array; an object array with a null run; message end."""
    b = bytearray()
    b += bytes([0]) + struct.pack("<4i", 1, -1, 1, 0)
    b += bytes([12]) + struct.pack("<i", 2) + _lps("Lib, Version=1.0.0.0")
    b += bytes([5]) + struct.pack("<i", 1) + _lps("NS.Thing") + struct.pack("<i", 4)
    b += _lps("count") + _lps("label") + _lps("data") + _lps("more")
    b += bytes([0, 1, 7, 5]) + bytes([8, 8])          # Primitive Int32, String, PrimitiveArray Int32, ObjectArray
    b += struct.pack("<i", 2)                         # library id
    b += struct.pack("<i", 42)                        # count
    b += bytes([6]) + struct.pack("<i", 3) + _lps("hi")   # label: BinaryObjectString
    b += bytes([9]) + struct.pack("<i", 4)            # data: MemberReference -> 4
    b += bytes([9]) + struct.pack("<i", 5)            # more: MemberReference -> 5
    b += bytes([15]) + struct.pack("<3i", 4, 3, 0)[:8] + bytes([8]) + struct.pack("<3i", 7, 8, 9)
    b += bytes([16]) + struct.pack("<2i", 5, 4) + bytes([9]) + struct.pack("<i", 3) + bytes([13, 2]) + bytes([10])
    b += bytes([11])
    root, end = nrbf.read(bytes(b))
    assert end == len(b)
    assert root.type_name == "NS.Thing" and root.library == "Lib, Version=1.0.0.0"
    assert root["count"] == 42 and root["label"] == "hi" and root["data"] == [7, 8, 9]
    assert root["more"] == ["hi", None, None, None]
    with pytest.raises(nrbf.NrbfError):
        nrbf.read(bytes(b[:-5]))


def test_nrbf_fragment_records():
    """The fragments' records as written: the List with its _items, a class
    record with member types for the first fragment and ClassWithId for the
    next, the faces as List<Int32> over a primitive array, and the role as
    an inline enum."""
    frags = [S.SurfaceFragment(id=4, faces=[1, 2], role=2), S.SurfaceFragment(id=5, faces=[], role=0)]
    blob = S._fragments_blob(frags)
    root, end = nrbf.read(blob)
    assert end == len(blob)
    assert root.type_name.startswith("System.Collections.Generic.List`1[[icFlow.SurfaceFragment, icFlowLibrary")
    items = nrbf.list_items(root)
    assert [o.member("<id>k__BackingField") for o in items] == [4, 5]
    assert items[0].member("<role>k__BackingField").type_name == "icFlow.SurfaceFragment+SurfaceRole"
    assert items[0]["faces"].type_name.startswith("System.Collections.Generic.List`1[[System.Int32, mscorlib")
    assert blob.count(bytes([nrbf.CLASS_WITH_ID])) >= 1
    assert S._fragments_from(root) == frags


def test_nrbf_rejects_bad_lengths():
    """Negative lengths and null runs past an array's end raise instead of
    allocating."""
    head = bytes([0]) + struct.pack("<4i", 1, -1, 1, 0)
    bad_prim = head + bytes([15]) + struct.pack("<2i", 1, -5) + bytes([8]) + bytes([11])
    bad_run = head + bytes([16]) + struct.pack("<2i", 1, 2) + bytes([14]) + struct.pack("<i", 1 << 30) + bytes([11])
    huge = head + bytes([16]) + struct.pack("<2i", 1, 1 << 30) + bytes([11])
    for b in (bad_prim, bad_run, huge):
        with pytest.raises(nrbf.NrbfError):
            nrbf.read(b)


@pytest.mark.parametrize("n", [1, 3, 4, 5, 300, 513])
def test_translation_lists_of_every_null_run(n):
    """TranslationCollection round trips whatever its capacity leaves empty:
    no nulls, one (ObjectNull), a short run (ObjectNullMultiple256) and a long
    one (ObjectNullMultiple)."""
    trans = [S.Translation(0.001 * i, -0.002 * i, 0.5, 1e-3 * i) for i in range(n)]
    blob = S._translations_blob(trans)
    root, end = nrbf.read(blob)
    assert end == len(blob)
    assert S._translations_from(root) == trans
    cap = max(4, 1 << (n - 1).bit_length())
    assert len(root.member("_items")) == cap
