"""Mesh files on the host (no GPU): OFF, TetGen and Medit parsing with the reference's
conventions (io/ParserOFF.cu, io/ParserTetGen.cu, io/ParserHex.cu) and the writers
(io/FileWriter.cu), round trips bit for bit, and the errors a caller sees."""
import numpy as np
import pytest

from volumesurfacediscretemeshoptimization_b200 import meshgen as G

TRI, QUAD, TET, HEX = 0, 1, 2, 3


def _rt(vsdmo, tmp_path, name, etype, xyz, el, fmt=0):
    p = str(tmp_path / name)
    vsdmo.write_mesh_file(p, etype, xyz, el, fmt)
    t, x2, e2 = vsdmo.read_mesh_file(p, fmt)
    assert t == etype
    assert np.array_equal(x2.view(np.uint32), np.asarray(xyz, np.float32).view(np.uint32))
    assert np.array_equal(e2, el)


def test_round_trips_are_bit_exact(vsdmo, tmp_path):
    xyz, tri = G.tri_grid(9, seed=1)
    xyz = xyz.copy()
    xyz[:, 2] = np.random.default_rng(0).standard_normal(len(xyz)).astype(np.float32) * 1e-3
    _rt(vsdmo, tmp_path, "a.off", TRI, xyz, tri)
    qx, quad = G.quad_grid(7, seed=2)
    _rt(vsdmo, tmp_path, "b.off", QUAD, qx, quad)
    tx, tet = G.tet_cube(3, seed=3)
    _rt(vsdmo, tmp_path, "c", TET, tx, tet)                   # TetGen base name
    _rt(vsdmo, tmp_path, "c2.node", TET, tx, tet)
    _rt(vsdmo, tmp_path, "d.mesh", TET, tx, tet)              # Medit tetrahedra
    hx, hexes = G.hex_cube(3, seed=4)
    _rt(vsdmo, tmp_path, "e.mesh", HEX, hx, hexes)
    _rt(vsdmo, tmp_path, "f.mesh", TRI, xyz, tri)


def test_hand_written_files(vsdmo, tmp_path):
    off = tmp_path / "q.off"
    off.write_text("OFF\n# a comment\n\n4 1 0\n0 0 0\n1 0 0 # trailing\n1 1 0\n0 1 0\n4 0 1 2 3 255 0 0\n")
    t, x, e = vsdmo.read_mesh_file(str(off))
    assert t == QUAD and x.shape == (4, 3) and e.tolist() == [[0, 1, 2, 3]]
    # TetGen, 1-based with attributes and boundary markers
    (tmp_path / "t.node").write_text("5 3 1 1\n1 0 0 0 7.5 1\n2 1 0 0 7.5 1\n3 0 1 0 7.5 1\n4 0 0 1 7.5 1\n"
                                     "5 .2 .2 .2 7.5 0\n")
    (tmp_path / "t.ele").write_text("# tets\n2 4 1\n1 1 2 3 5 9\n2 1 2 4 5 9\n")
    t, x, e = vsdmo.read_mesh_file(str(tmp_path / "t"))
    assert t == TET and len(x) == 5 and e.tolist() == [[0, 1, 2, 4], [0, 1, 3, 4]]
    assert abs(x[4, 0] - 0.2) < 1e-7
    # Medit hexahedron: file corners (bottom face first) are stored with the faces swapped
    pts = "\n".join(f"{i % 2} {(i // 2) % 2} {i // 4} 0" for i in range(8))
    (tmp_path / "h.mesh").write_text("MeshVersionFormatted 1\nDimension 3\nVertices 8\n" + pts +
                                     "\nHexahedra 1\n1 2 4 3 5 6 8 7 0\nEnd\n")
    t, x, e = vsdmo.read_mesh_file(str(tmp_path / "h.mesh"))
    assert t == HEX and e.tolist() == [[4, 5, 7, 6, 0, 1, 3, 2]]
    # Medit, 2D vertices and triangles
    (tmp_path / "p.mesh").write_text("MeshVersionFormatted 2\nDimension 2\nVertices 3\n0 0 1\n1 0 1\n0 1 1\n"
                                     "Edges 1\n1 2 0\nTriangles 1\n1 2 3 0\nEnd\n")
    t, x, e = vsdmo.read_mesh_file(str(tmp_path / "p.mesh"))
    assert t == TRI and x[:, 2].tolist() == [0, 0, 0] and e.tolist() == [[0, 1, 2]]


@pytest.mark.parametrize("name,text,msg", [
    ("bad1.off", "COFF\n3 1 0\n0 0 0\n1 0 0\n0 1 0\n3 0 1 2\n", b"not OFF"),
    ("bad2.off", "OFF\n3 1 0\n0 0 0\n1 0 0\n0 1 0\n3 0 1 5\n", b"out of range"),
    ("bad3.off", "OFF\n4 2 0\n0 0 0\n1 0 0\n0 1 0\n1 1 0\n3 0 1 2\n4 0 1 3 2\n", b"mixed"),
    ("bad4.mesh", "MeshVersionFormatted 1\nDimension 3\nVertices 9\n" + "0 0 0 0\n" * 9 +
     "Hexahedra 1\n1 2 3 4 5 6 7 8 0\nEnd\n", b"no hexahedron uses"),
    ("bad5.mesh", "MeshVersionFormatted 1\nDimension 3\nCorners 1\n1\nEnd\n", b"unsupported section"),
    ("bad6.off", "OFF\n3 1 0\n0 0 0\n1 0 0\n", b"missing vertex"),
])
def test_parse_errors(vsdmo, tmp_path, name, text, msg):
    (tmp_path / name).write_text(text)
    with pytest.raises(vsdmo.VSDMOError) as ei:
        vsdmo.read_mesh_file(str(tmp_path / name))
    assert ei.value.status == vsdmo._capi.E_IO
    assert msg in vsdmo._capi.lib().vsdmo_last_error()


def test_missing_file_and_format(vsdmo, tmp_path):
    with pytest.raises(vsdmo.VSDMOError) as ei:
        vsdmo.read_mesh_file(str(tmp_path / "nope.off"))
    assert ei.value.status == vsdmo._capi.E_IO
    with pytest.raises(vsdmo.VSDMOError):
        vsdmo.read_mesh_file(str(tmp_path / "unknown.xyz"))
    # OFF holds surfaces only
    tx, tet = G.tet_cube(2, seed=1)
    with pytest.raises(vsdmo.VSDMOError):
        vsdmo.write_mesh_file(str(tmp_path / "t.off"), TET, tx, tet)
    # a factory returns None for a missing file, like the reference's nullptr
    assert vsdmo.DMOMeshTetFactory.create(str(tmp_path / "missing")) is None
