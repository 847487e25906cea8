"""Invalid inputs through the C ABI: the build checks the element indices and coordinates
before it uses them and detects non-manifold fans during the fan walk (bounded by the row
length), so each case ends in a status, never a device fault; the library stays usable after
it. The oracle rejects the same meshes (oracle/or_conn.c)."""
import numpy as np
import pytest

from volumesurfacediscretemeshoptimization_b200 import meshgen as G

pytestmark = pytest.mark.gpu
TRI, TET = 0, 2


def _status(vsdmo, fn):
    with pytest.raises(vsdmo.VSDMOError) as e:
        fn()
    return e.value.status


def test_invalid_tet_meshes(vsdmo, oracle_mod):
    from volumesurfacediscretemeshoptimization_b200 import _capi
    xyz, tets = G.tet_cube(3, seed=1)
    bad_index = np.vstack([tets, [[0, 1, 2, len(xyz)]]]).astype(np.int32)
    assert _status(vsdmo, lambda: vsdmo.DMOMeshTet(xyz, bad_index)) == _capi.E_ARG
    neg_index = np.vstack([tets, [[0, 1, 2, -1]]]).astype(np.int32)
    assert _status(vsdmo, lambda: vsdmo.DMOMeshTet(xyz, neg_index)) == _capi.E_ARG
    nan_xyz = xyz.copy()
    nan_xyz[5, 1] = np.nan
    assert _status(vsdmo, lambda: vsdmo.DMOMeshTet(nan_xyz, tets)) == _capi.E_NAN
    inf_xyz = xyz.copy()
    inf_xyz[7, 2] = np.inf
    assert _status(vsdmo, lambda: vsdmo.DMOMeshTet(inf_xyz, tets)) == _capi.E_NAN
    dup = np.vstack([tets, tets[:1]]).astype(np.int32)
    assert _status(vsdmo, lambda: vsdmo.DMOMeshTet(xyz, dup)) == _capi.E_NONMANIFOLD
    with pytest.raises(Exception):
        oracle_mod.OracleMesh(TET, xyz, dup)
    # the library is still usable
    gm = vsdmo.DMOMeshTet(xyz, tets)
    opt = vsdmo.DMOTetClass(gm, n_iter=2)
    q0 = opt.getQuality()
    opt.optimize()
    assert opt.getQuality() > q0


def test_invalid_triangle_meshes(vsdmo, oracle_mod):
    from volumesurfacediscretemeshoptimization_b200 import _capi
    xyz, tri = G.tri_grid(6, seed=1)
    dup = np.vstack([tri, tri[:1]]).astype(np.int32)
    assert _status(vsdmo, lambda: vsdmo.DMOMeshTri(xyz, dup)) == _capi.E_NONMANIFOLD
    flip = np.vstack([tri[:-1], tri[-1:, ::-1]]).astype(np.int32)
    assert _status(vsdmo, lambda: vsdmo.DMOMeshTri(xyz, flip)) == _capi.E_NONMANIFOLD
    for el in (dup, flip):
        with pytest.raises(Exception):
            oracle_mod.OracleMesh(TRI, xyz, el)
    bad = tri.copy()
    bad[3, 1] = len(xyz) + 5
    assert _status(vsdmo, lambda: vsdmo.DMOMeshTri(xyz, bad)) == _capi.E_ARG
    gm = vsdmo.DMOMeshTri(xyz, tri)
    vsdmo.DMOTriFlatClass(gm, n_iter=1).optimize()


def test_invalid_optimiser_parameters(vsdmo):
    from volumesurfacediscretemeshoptimization_b200 import _capi
    xyz, tets = G.tet_cube(3, seed=1)
    gm = vsdmo.DMOMeshTet(xyz, tets)
    for kw in ({"depth": 0}, {"depth": 9}, {"gridScale": -0.5}, {"gridScale": float("nan")}, {"n_iter": -1},
               {"fit_ring": 3}, {"grid_n": 5}):
        st = _status(vsdmo, lambda: vsdmo.DMOTetClass(gm, **kw))
        assert st in (_capi.E_ARG, _capi.E_UNSUPPORTED), kw
    opt = vsdmo.DMOTetClass(gm, n_iter=1)
    assert _status(vsdmo, lambda: opt.run_color(10 ** 6)) == _capi.E_ARG
    assert _status(vsdmo, lambda: opt.getLocalSurfacePoints(0, 4, 4)) == _capi.E_ARG
