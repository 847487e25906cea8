"""GPU tests of the angle criteria (MIN_ANGLE / MAX_ANGLE) in the surface, sliding-boundary and
volume-boundary passes: DMOTriFlatClass with sliding boundary vertices (the reference class's
default criterion is MIN_ANGLE), DMOTriClass on a surface with feature lines, DMOTetClass with
a free boundary. One iteration against the oracle's literal double restatement
(oracle/or_dmo.c, or_surf.c, or_feat.c, or_vring.c under oracle.criterion) within 1e-5 h
wherever the double decisions are clear by more than 2e-5 (CUDA's acosf is not the host's
acos, so there is no bitwise check), element qualities within 2e-5, and the known answers:
boundary vertices stay on their lines / faces / edges and the minimum quality never drops."""
import numpy as np
import pytest

from volumesurfacediscretemeshoptimization_b200 import meshgen as G
from test_gpu_features import cube_surface_with_jitter, square_with_boundary_jitter
from test_gpu_volume_boundary import jittered_cube

pytestmark = pytest.mark.gpu
TRI, TET = 0, 2
CLEAR = 2e-5
CRITS = ["MIN_ANGLE", "MAX_ANGLE"]


def _clear_ring(clear, rp, nb, v0, v1):
    """a vertex is comparable only when the vertices its search reads are"""
    for v in range(v0, v1):
        clear[v] &= bool(np.all(clear[nb[rp[v]:rp[v + 1]].ravel()]))


def _crit(oracle_mod, vsdmo, name):
    return getattr(vsdmo.QualityCriterium, name), getattr(oracle_mod, name), name == "MAX_ANGLE"


@pytest.mark.parametrize("name", CRITS)
def test_flat_sliding_boundary_angle(oracle_mod, vsdmo, name):
    c, oc, mx = _crit(oracle_mod, vsdmo, name)
    n = 16
    h = 1.0 / (n - 1)
    xyz, tri = square_with_boundary_jitter(n, seed=2)
    om = oracle_mod.OracleMesh(TRI, xyz, tri)
    gm = vsdmo.DMOMeshTri(xyz, tri)
    opt = vsdmo.DMOTriFlatClass(gm, qualityCriterium=c, n_iter=1, fix_boundary=False)
    x = om.xyz.astype(np.float64)
    assert om.angle_qualities_f64(x, mx).min() > 0
    clear = np.ones(len(x), bool)
    rp = om.array(oracle_mod.A_HE_ROWPTR)
    he = om.array(oracle_mod.A_HALFEDGES).reshape(-1, 4)[:, 0]
    for v0, v1 in om.color_ranges():
        x, mg = om.dmo_angle_f64(x, v0, v1, mx)
        clear[v0:v1] &= mg > CLEAR
        _clear_ring(clear, rp, he, v0, v1)
    vn = np.zeros_like(x); vn[:, 2] = 1
    fdeg, flags = om.feature_flags(om.xyz)
    curves = om.curves_f64(om.xyz.astype(np.float64), vn)
    nn = np.arange(len(x), dtype=np.int32)
    cf = om.array(oracle_mod.A_COL_FEATURE)
    with oracle_mod.criterion(oc):
        for k in range(len(cf) - 1):
            v0, v1 = int(cf[k]), int(cf[k + 1])
            x, mg = om.dmo_1d_f64(x, om.xyz, curves, nn, vn, fdeg, flags, v0, v1)
            clear[v0:v1] &= mg > CLEAR
            _clear_ring(clear, rp, he, v0, v1)
    opt.iterate(1)
    g = gm.positions().astype(np.float64)
    d = np.abs(g - x)[:, :2].max(1)
    assert np.all(d[clear] < 1e-5 * h), float(d[clear].max())
    nFree = om.info["nSurf"] - om.info["nFeature"]
    # a boundary vertex sliding on a line sees the angles at its line neighbours unchanged for
    # every candidate: those exact ties leave a part of the boundary decisions open
    assert clear[:nFree].sum() > 0.6 * nFree and clear[nFree:].sum() > 0.15 * (len(x) - nFree)
    assert np.any(x[nFree:] != om.xyz[nFree:])
    # known answers over more iterations: boundary vertices stay on the square's lines, the
    # minimum never drops
    opt2 = vsdmo.DMOTriFlatClass(vsdmo.DMOMeshTri(xyz, tri), qualityCriterium=c, n_iter=5, fix_boundary=False)
    opt2.optimize()
    g2 = opt2.mesh.positions(original_order=True)
    for i, p0 in enumerate(xyz):
        for a in range(2):
            if p0[a] in (0.0, 1.0):
                assert abs(g2[i, a] - p0[a]) < 1e-6
    mn, _ = opt2.history()
    assert np.all(np.diff(mn) >= -1e-6) and mn[-1] > mn[0]


@pytest.mark.parametrize("name", CRITS)
def test_surface_angle_with_features(oracle_mod, vsdmo, name):
    c, oc, mx = _crit(oracle_mod, vsdmo, name)
    sx, faces = cube_surface_with_jitter(vsdmo)
    h = 1.0 / 5
    om = oracle_mod.OracleMesh(TRI, sx, faces)
    gm = vsdmo.DMOMeshTri(sx, faces)
    opt = vsdmo.DMOTriClass(gm, qualityCriterium=c, n_iter=1)
    with oracle_mod.criterion(oc):
        np.testing.assert_allclose(opt.getElementQualities(), om.element_qualities_f64(gm.positions().astype(np.float64)),
                                   rtol=0, atol=2e-5)
        x32 = om.xyz
        x = x32.astype(np.float64)
        x0, ls, nn, vn = om.surface_state_f64(x32)
        fn = om.array(oracle_mod.A_FACE_NORMALS).reshape(-1, 3).astype(np.float64)
        sectors = om.sector_surfaces(x32, fn, dtype=np.float64)
        rp = om.array(oracle_mod.A_HE_ROWPTR)
        he = om.array(oracle_mod.A_HALFEDGES).reshape(-1, 4)[:, 0]
        clear = np.ones(len(x), bool)
        for v0, v1 in om.color_ranges():
            x, mg = om.dmo_surf_feat_f64(x, x0, ls, nn, vn, sectors, v0, v1)
            clear[v0:v1] &= mg > CLEAR
            _clear_ring(clear, rp, he, v0, v1)
        fdeg, flags = om.feature_flags(x32)
        curves = om.curves_f64(x32, vn)
        cf = om.array(oracle_mod.A_COL_FEATURE)
        for k in range(len(cf) - 1):
            v0, v1 = int(cf[k]), int(cf[k + 1])
            x, mg = om.dmo_1d_f64(x, x0, curves, nn, vn, fdeg, flags, v0, v1)
            clear[v0:v1] &= mg > CLEAR
            _clear_ring(clear, rp, he, v0, v1)
    opt.iterate(1)
    d = np.abs(gm.positions().astype(np.float64) - x).max(1)
    assert np.all(d[clear] < 1e-5 * h), float(d[clear].max())
    assert clear.sum() > 0.5 * len(x) and np.any(x != x32)
    # face vertices stay in their face planes. (Edge vertices need not stay on their edges:
    # once one slides nearer to an initial vertex next to a corner, whose curve is fitted
    # through feature vertices of two edges, the reference's curve of the nearest initial
    # vertex bends it off the edge -- the optimiser reproduces that.)
    opt2 = vsdmo.DMOTriClass(vsdmo.DMOMeshTri(sx, faces), qualityCriterium=c, n_iter=4)
    opt2.optimize()
    g = opt2.mesh.positions(original_order=True)
    for i, p0 in enumerate(sx):
        on = (np.abs(p0) < 1e-7) | (np.abs(p0 - 1) < 1e-7)
        if on.sum() == 1:
            assert np.all(np.abs(g[i, on] - p0[on]) < 1e-6), (i, p0, g[i])
    mn, _ = opt2.history()
    assert np.all(np.diff(mn) >= -1e-6) and mn[-1] > mn[0]


@pytest.mark.parametrize("name", CRITS)
def test_tet_boundary_angle(oracle_mod, vsdmo, name):
    """The boundary passes class by class from the product's own input state, in double: each
    boundary class moves only its own vertices, so the state a class saw is the product's
    final positions for the interior and the classes before it and the positions after the
    interior classes (an iteration with the boundary held runs the same interior launches on the
    same input) for the classes after it. Angle rings tie exactly along sliding lines, and a tie
    that is exact in one state can become a near-tie under the other's rounding, so the
    comparison is per class, not along a double run of the whole pass."""
    c, oc, mx = _crit(oracle_mod, vsdmo, name)
    xyz, el, h = jittered_cube("tet")
    om = oracle_mod.OracleMesh(TET, xyz, el)
    x32 = om.xyz
    assert om.angle_qualities_f64(x32.astype(np.float64), mx).min() > 0
    held = vsdmo.DMOMeshTet(xyz, el)
    vsdmo.DMOTetClass(held, qualityCriterium=c, n_iter=1).iterate(1)
    xi = held.positions()
    gm = vsdmo.DMOMeshTet(xyz, el)
    opt = vsdmo.DMOTetClass(gm, qualityCriterium=c, n_iter=1, fix_boundary=False)
    opt.iterate(1)
    g = gm.positions()
    nS = om.info["nSurf"]
    assert np.array_equal(g[nS:], xi[nS:]) and np.array_equal(xi[:nS], x32[:nS])
    clear = np.zeros(nS, bool)
    x = np.zeros((nS, 3))

    def ranges(a):
        arr = om.array(a)
        return [(int(arr[i]), int(arr[i + 1])) for i in range(len(arr) - 1)]

    classes = ranges(oracle_mod.A_COL_FREE) + ranges(oracle_mod.A_COL_FEATURE)
    n_free = len(ranges(oracle_mod.A_COL_FREE))

    def seen(k):
        """the state boundary class k read: the product's positions, later classes not yet moved"""
        st = g.astype(np.float64).copy()
        for v0, v1 in classes[k:]:
            st[v0:v1] = xi[v0:v1]
        return st

    x0, ls, nn, vn = om.surface_state_f64(x32)
    fn = om.array(oracle_mod.A_FACE_NORMALS).reshape(-1, 3).astype(np.float64)
    sectors = om.sector_surfaces(x32, fn, dtype=np.float64)
    with oracle_mod.criterion(oc):
        fdeg, flags = om.feature_flags(x32)
        curves = om.curves_f64(x32, vn)
        for k, (v0, v1) in enumerate(classes):
            if k < n_free:
                y, mg = om.dmo_vol_surf_f64(seen(k), x0, ls, nn, sectors, v0, v1)
            else:
                y, mg = om.dmo_1d_f64(seen(k), x0, curves, nn, vn, fdeg, flags, v0, v1)
            x[v0:v1] = y[v0:v1]
            clear[v0:v1] = mg > CLEAR
    d = np.abs(g[:nS].astype(np.float64) - x).max(1)
    assert np.all(d[clear] < 1e-5 * h), float(d[clear].max())
    assert clear.sum() > 0.2 * nS and np.any(x != x32[:nS])
    opt2 = vsdmo.DMOTetClass(vsdmo.DMOMeshTet(xyz, el), qualityCriterium=c, n_iter=3, fix_boundary=False)
    opt2.optimize()
    g = opt2.mesh.positions(original_order=True)
    for i, p0 in enumerate(xyz):
        on = (np.abs(p0) < 1e-7) | (np.abs(p0 - 1) < 1e-7)
        assert np.all(np.abs(g[i, on] - p0[on]) < 1e-6), (i, p0, g[i])
    mn, _ = opt2.history()
    assert np.all(np.diff(mn) >= -1e-6) and mn[-1] > mn[0]

