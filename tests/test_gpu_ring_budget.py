"""Rings at and over the kernels' shared-memory budgets (the reference stages one-rings in
dynamic shared memory sized by the largest ring, DMOTetImplCub.h:21-60, DMOTriFlatImplCub.h:
24-85). A vertex whose ring fills the budget exactly is optimised bit for bit like the oracle
does; one element more and creating the optimiser ends in VSDMO_E_VALENCE, never a launch with
an overflowing ring. The library stays usable after it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TRI, TET = 0, 2
TET_RING_BUDGET = 512      # tetrahedra around one vertex (dmo_tet_max_ring)
FLAT_RING_BUDGET = 256     # halfedges out of one vertex, 8x8 flat search (dmo_tri2d_max_ring)
SLIDE_RING_BUDGET = 64     # the same with sliding boundaries, whose passes run the surface kernels


def _uv_sphere(n_lon, n_lat):
    """Closed UV sphere: poles, n_lat - 1 rings of n_lon vertices, 2 n_lon (n_lat - 1) triangles."""
    v = [[0.0, 0.0, 1.0]]
    for i in range(1, n_lat):
        th = np.pi * i / n_lat
        for j in range(n_lon):
            ph = 2 * np.pi * j / n_lon
            v.append([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])
    v.append([0.0, 0.0, -1.0])
    ring = lambda i, j: 1 + (i - 1) * n_lon + (j % n_lon)
    t = [[0, ring(1, j), ring(1, j + 1)] for j in range(n_lon)]
    for i in range(1, n_lat - 1):
        for j in range(n_lon):
            a, b, c, d = ring(i, j), ring(i + 1, j), ring(i + 1, j + 1), ring(i, j + 1)
            t += [[a, b, c], [a, c, d]]
    s = len(v) - 1
    t += [[s, ring(n_lat - 1, j + 1), ring(n_lat - 1, j)] for j in range(n_lon)]
    return np.array(v), np.array(t)


def tet_star(n_tets):
    """One interior vertex (off centre) joined to every triangle of a closed sphere."""
    n_lon = 16
    sv, st = _uv_sphere(n_lon, n_tets // (2 * n_lon) + 1)
    assert len(st) == n_tets
    c = len(sv)
    xyz = np.vstack([sv, [[0.11, -0.07, 0.05]]]).astype(np.float32)
    tets = np.hstack([np.full((len(st), 1), c), st])
    p = xyz[tets].astype(np.float64)
    det = np.linalg.det(np.stack([p[:, 1] - p[:, 0], p[:, 2] - p[:, 0], p[:, 3] - p[:, 0]], axis=1))
    tets[det < 0] = tets[det < 0][:, [0, 2, 1, 3]]
    return xyz, tets.astype(np.int32)


def tri_fan(k):
    """One interior vertex (off centre) joined to the k edges of a regular k-gon."""
    a = 2 * np.pi * np.arange(k) / k
    xyz = np.zeros((k + 1, 3), np.float32)
    xyz[:k, 0], xyz[:k, 1] = np.cos(a), np.sin(a)
    xyz[k] = [0.13, -0.09, 0.0]
    tris = np.array([[k, i, (i + 1) % k] for i in range(k)], np.int32)
    return xyz, tris


def _colour_launches_bitwise(om, gm, opt):
    x = om.xyz
    assert np.array_equal(gm.positions(), x)
    moved = 0
    for c, (v0, v1) in enumerate(om.color_ranges()):
        x_next = om.dmo_color_f32(x, v0, v1)
        opt.run_color(c)
        g = gm.positions()
        assert np.array_equal(g.view(np.uint32), x_next.view(np.uint32)), c
        moved += int(np.any(x_next != x, axis=1).sum())
        x = x_next
    return moved


def test_tet_ring_at_budget_is_bitwise(oracle_mod, vsdmo):
    xyz, tets = tet_star(TET_RING_BUDGET)
    gm = vsdmo.DMOMeshTet(xyz, tets)
    assert gm.info["maxNumTetrahedra"] == TET_RING_BUDGET
    om = oracle_mod.OracleMesh(TET, xyz, tets)
    opt = vsdmo.DMOTetClass(gm, vsdmo.QualityCriterium.MEAN_RATIO, 0.5, 2)
    q0 = opt.getQuality()
    assert _colour_launches_bitwise(om, gm, opt) == 1
    assert opt.findMinimumQuality() > q0


def test_tet_ring_over_budget_is_refused(vsdmo):
    from volumesurfacediscretemeshoptimization_b200 import _capi
    xyz, tets = tet_star(TET_RING_BUDGET + 32)
    gm = vsdmo.DMOMeshTet(xyz, tets)
    with pytest.raises(vsdmo.VSDMOError) as e:
        vsdmo.DMOTetClass(gm)
    assert e.value.status == _capi.E_VALENCE
    xyz, tets = tet_star(TET_RING_BUDGET)
    opt = vsdmo.DMOTetClass(vsdmo.DMOMeshTet(xyz, tets), n_iter=2)
    q0 = opt.getQuality()
    opt.optimize()
    assert opt.getQuality() > q0


def test_flat_ring_at_budget_is_bitwise(oracle_mod, vsdmo):
    xyz, tris = tri_fan(FLAT_RING_BUDGET)
    gm = vsdmo.DMOMeshTri(xyz, tris)
    assert gm.info["maxNumHalfedges"] == FLAT_RING_BUDGET
    om = oracle_mod.OracleMesh(TRI, xyz, tris)
    opt = vsdmo.DMOTriFlatClass(gm, vsdmo.QualityCriterium.MEAN_RATIO, 0.5, 2)
    q0 = opt.getQuality()
    assert _colour_launches_bitwise(om, gm, opt) == 1
    assert opt.findMinimumQuality() > q0


def test_flat_ring_over_budget_is_refused(vsdmo):
    from volumesurfacediscretemeshoptimization_b200 import _capi
    for k, fix in ((FLAT_RING_BUDGET + 1, True), (SLIDE_RING_BUDGET + 1, False)):
        xyz, tris = tri_fan(k)
        gm = vsdmo.DMOMeshTri(xyz, tris)
        with pytest.raises(vsdmo.VSDMOError) as e:
            vsdmo.DMOTriFlatClass(gm, fix_boundary=fix)
        assert e.value.status == _capi.E_VALENCE, (k, fix)
    # at the sliding budget the boundary vertices slide and the run stays monotone
    xyz, tris = tri_fan(SLIDE_RING_BUDGET)
    opt = vsdmo.DMOTriFlatClass(vsdmo.DMOMeshTri(xyz, tris), n_iter=2, fix_boundary=False)
    q0 = opt.getQuality()
    opt.optimize()
    assert opt.getQuality() >= q0
