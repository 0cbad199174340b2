"""Gmsh 2.2 import and export (v3Library/Geometry/Mesh/Mesh.cs:548-616)."""
import io

import numpy as np
import pytest

from icflow_b200 import mesh as M
from icflow_b200 import mesh_io


def _grains_mesh(n=4, grains=5, seed=3):
    m = M.box_mesh((n, n, n), (1e-3, 1e-3, 1e-3), name="cube")
    g = M.voronoi_grains(m.x0, m.elems, grains, seed)
    return m, g


def test_round_trip_keeps_nodes_tets_and_grains(tmp_path):
    m, g = _grains_mesh()
    p = tmp_path / "cube.msh"
    mesh_io.write_msh(p, m.x0, m.elems, g, triangles=m.faces)
    d = mesh_io.read_msh(p)
    assert np.array_equal(d.x0, m.x0)  # repr() of a double reads back exactly
    assert np.array_equal(d.elems, m.elems) and np.array_equal(d.granule, g)
    assert np.array_equal(d.triangles, m.faces)


def test_loaded_mesh_gets_the_same_czs_as_the_generator(tmp_path):
    m, g = _grains_mesh()
    ref = M.insert_czs(m, g)
    buf = io.StringIO()
    mesh_io.write_msh(buf, m.x0, m.elems, g)
    got = mesh_io.load_msh(buf.getvalue(), name="cube")
    for f in ("x0", "elems", "czs", "faces", "face_exposed", "cz_faces"):
        assert np.array_equal(getattr(got, f), getattr(ref, f)), f
    assert got.name == "cube" and got.isDeformable
    # a one-grain file has no CZs
    buf = io.StringIO()
    mesh_io.write_msh(buf, m.x0, m.elems)
    one = mesh_io.load_msh(buf.getvalue())
    assert len(one.czs) == 0 and np.array_equal(one.elems, m.elems)


def test_reads_the_reference_layout_with_points_lines_and_triangles():
    # the reference's files: three tags per element, node fields from the
    # seventh on, point (15), line (1), triangle (2) and tet (4) records
    text = "\n".join([
        "$MeshFormat", "2.2 0 8", "$EndMeshFormat",
        "$Nodes", "5",
        "1 0 0 0", "2 1 0 0", "3 0 1 0", "4 0 0 1", "5 1 1 1",
        "$EndNodes",
        "$Elements", "5",
        "1 15 3 0 1 0 1",
        "2 1 3 0 7 0 1 2",
        "3 2 3 0 9 0 1 2 3",
        "4 4 3 0 1 0 1 2 3 4",
        "5 4 3 0 2 0 2 3 4 5",
        "$EndElements", ""])
    d = mesh_io.read_msh(text)
    assert d.x0.shape == (5, 3)
    assert np.array_equal(d.elems, [[0, 1, 2, 3], [1, 2, 3, 4]])
    assert np.array_equal(d.granule, [0, 1])
    assert np.array_equal(d.triangles, [[0, 1, 2]]) and np.array_equal(d.edges, [[0, 1]])
    m = mesh_io.load_msh(text)
    assert len(m.czs) == 1  # the shared face of the two grains


@pytest.mark.parametrize("bad", [
    "$Nodes\n2\n1 0 0 0\n$EndNodes\n$Elements\n0\n$EndElements\n",  # count mismatch
    "$Nodes\n1\n1 0 0 0\n$EndNodes\n$Elements\n1\n1 4 3 0 1 0 1 2 3 4\n$EndElements\n",  # node out of range
    "no mesh here\n",
])
def test_malformed_files_are_rejected(bad):
    with pytest.raises(ValueError):
        mesh_io.read_msh(bad)
