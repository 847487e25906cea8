"""GPU side of the mesh files and the surface factories: a mesh created from a file is the
mesh created from the same arrays (connectivity and colouring bit-exact), an optimised mesh
written and read back carries its positions bit for bit in the caller's numbering, and the
boundary surface of a volume mesh (DMOMeshTriFactory::create(DMOMeshTet&),
DMOMeshQuadFactory::create(DMOMeshHex&)) matches the oracle's build of the same arrays."""
import numpy as np
import pytest

from volumesurfacediscretemeshoptimization_b200 import meshgen as G

pytestmark = pytest.mark.gpu
TRI, QUAD, TET, HEX = 0, 1, 2, 3


@pytest.mark.parametrize("etype,name", [(TET, "cube"), (HEX, "cube.mesh"), (TRI, "grid.off"), (QUAD, "q.off")])
def test_file_mesh_equals_array_mesh(vsdmo, tmp_path, etype, name):
    gen = {TET: lambda: G.tet_cube(6, seed=1), HEX: lambda: G.hex_cube(5, seed=2),
           TRI: lambda: G.tri_grid(20, seed=3), QUAD: lambda: G.quad_grid(15, seed=4)}[etype]
    xyz, el = gen()
    path = str(tmp_path / name)
    vsdmo.write_mesh_file(path, etype, xyz, el)
    fac = {TET: vsdmo.DMOMeshTetFactory, HEX: vsdmo.DMOMeshHexFactory, TRI: vsdmo.DMOMeshTriFactory,
           QUAD: vsdmo.DMOMeshQuadFactory}[etype]
    a = fac.create(path)
    b = fac.create(xyz, el)
    assert a.info == b.info
    A, B = a.arrays(), b.arrays()
    for k in A:
        assert np.array_equal(A[k].view(np.uint8), B[k].view(np.uint8)), k


def test_optimised_mesh_written_and_read_back(vsdmo, tmp_path):
    xyz, tets = G.tet_cube(8, seed=5)
    mesh = vsdmo.DMOMeshTet(xyz, tets)
    opt = vsdmo.DMOTetClass(mesh, n_iter=3)
    opt.optimize()
    for name in ("out", "out.mesh"):
        path = str(tmp_path / name)
        mesh.write(path)
        t, x, e = vsdmo.read_mesh_file(path)
        assert t == TET and np.array_equal(e, tets)
        assert np.array_equal(x.view(np.uint32), mesh.positions(original_order=True).view(np.uint32))
    # a wrong factory for the file's element type is an error, not a garbage mesh
    with pytest.raises(vsdmo.VSDMOError):
        vsdmo.DMOMeshHexFactory.create(str(tmp_path / "out.mesh"))


@pytest.mark.parametrize("etype", [TET, HEX])
def test_boundary_surface_factory(oracle_mod, vsdmo, etype):
    if etype == TET:
        xyz, el = G.tet_cube(7, seed=6)
        vol = vsdmo.DMOMeshTet(xyz, el)
        surf = vsdmo.DMOMeshTriFactory.create(vol)
        k, st = 3, TRI
    else:
        xyz, el = G.hex_cube(6, seed=7)
        vol = vsdmo.DMOMeshHex(xyz, el)
        surf = vsdmo.DMOMeshQuadFactory.create(vol)
        k, st = 4, QUAD
    nS = vol.info["nSurf"]
    assert surf.info["nV"] == nS and surf.info["nE"] == vol.info["nTris"]
    sx = vol.positions()[:nS]
    faces = vol.array(vsdmo.A_SURF_TRIS).reshape(-1, k)
    om = oracle_mod.OracleMesh(st, sx, faces)
    assert om.info == surf.info
    A = om.arrays()
    B = surf.arrays()
    for key in ("new_of_old", "halfedges", "he_rowptr", "col_free", "is_feature"):
        assert np.array_equal(A[key], B[key]), key
