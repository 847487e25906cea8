"""GPU parity tests of the feature / boundary passes: the 1D pass of flat meshes with sliding
boundaries (k_optimizeHierarchical1DFlat) and of surfaces with feature lines
(k_optimizeHierarchical1D), the curves and 1D flags, the per-sector surfaces of feature
vertices and the feature-aware surface estimate of the free vertices — bitwise against the
oracle's f32 restatement (oracle/or_feat.c, oracle/or_surf.c) over whole iterations, within the
FP64 restatement's tolerance, and the known answers of straight boundaries and flat faces:
vertices stay on them."""
import ctypes as C

import numpy as np
import pytest

from volumesurfacediscretemeshoptimization_b200 import meshgen as G

pytestmark = pytest.mark.gpu
TRI, QUAD = 0, 1


def same_bits(a, b):
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape:
        return False
    na, nb = np.isnan(a), np.isnan(b)
    return bool(np.array_equal(na, nb) and np.array_equal(a[~na].view(np.uint32), b[~nb].view(np.uint32)))


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def square_with_boundary_jitter(n=16, seed=2):
    """Flat triangle grid on the unit square, interior jitter 0.4h and boundary vertices
    displaced along their boundary line by up to 0.3h (corners fixed)."""
    h = 1.0 / (n - 1)
    xyz, tri = G.tri_grid(n, seed=seed, jitter=0.4)
    xyz = xyz.astype(np.float64)
    rng = np.random.default_rng(seed + 100)
    for i in range(len(xyz)):
        x, y = xyz[i, :2]
        if (abs(y) < 1e-9 or abs(y - 1) < 1e-9) and 1e-9 < x < 1 - 1e-9:
            xyz[i, 0] += rng.uniform(-0.3 * h, 0.3 * h)
        if (abs(x) < 1e-9 or abs(x - 1) < 1e-9) and 1e-9 < y < 1 - 1e-9:
            xyz[i, 1] += rng.uniform(-0.3 * h, 0.3 * h)
    return xyz.astype(np.float32), tri


def cube_surface_with_jitter(vsdmo, n=5, seed=3, quads=False):
    """Boundary surface of an undistorted tet (hex) cube with every surface vertex displaced
    within its face plane / along its edge (corners fixed): the surface stays the cube."""
    if quads:
        xyz, el = G.hex_cube(n, seed=None)
        vol = vsdmo.DMOMeshHex(xyz, el)
    else:
        xyz, el = G.tet_cube(n, seed=None)
        vol = vsdmo.DMOMeshTet(xyz, el)
    nS = vol.info["nSurf"]
    sx = vol.positions()[:nS].astype(np.float64)
    faces = vol.array(vsdmo.A_SURF_TRIS).reshape(-1, 4 if quads else 3)
    h = 1.0 / n
    rng = np.random.default_rng(seed)
    for i in range(nS):
        on = (np.abs(sx[i]) < 1e-9) | (np.abs(sx[i] - 1) < 1e-9)
        for a in range(3):
            if not on[a] and on.sum() < 3:
                sx[i, a] += rng.uniform(-0.25 * h, 0.25 * h)
    return sx.astype(np.float32), faces


def _oracle_iteration(oracle_mod, om, x, state, slide, sectors):
    """One iteration of the reference loop on the oracle (f32); state = dict(x0, ls, nn, vn, fn,
    curves, fdeg, opt). Flat meshes run the 1D pass only while the minimum quality after the
    previous iteration is positive (dmo/DMOTriFlat.cu:140)."""
    L = oracle_mod.lib()
    gate = om.element_qualities_f32(x).min() > 0 if slide else True
    for (v0, v1) in om.color_ranges():
        if slide:
            x = om.dmo_color_f32(x, v0, v1)
        elif sectors is not None:
            x = om.dmo_surf_feat_f32(x, state["x0"], state["ls"], state["nn"], state["vn"], sectors, v0, v1)
        else:
            x = om.dmo_surf_color_f32(x, (state["x0"], state["ls"], state["nn"], None, state["vn"]), v0, v1)
    cf = om.array(oracle_mod.A_COL_FEATURE)
    if gate:
        for c in range(len(cf) - 1):
            x = om.dmo_1d_f32(x, state["x0"], state["curves"], state["nn"], state["vn"], state["fdeg"], state["opt"],
                              int(cf[c]), int(cf[c + 1]))
    nn = state["nn"].copy()
    L.or_update_nn_f32(om.h, _p(np.ascontiguousarray(x, np.float32)), _p(state["x0"]), _p(nn))
    state["nn"] = nn
    if not slide:
        fn = np.zeros_like(state["fn"]); vn = np.zeros_like(state["vn"])
        L.or_surface_normals_f32(om.h, _p(np.ascontiguousarray(x, np.float32)), _p(fn), _p(vn))
        state["fn"], state["vn"] = fn, vn
    return x


def test_flat_sliding_boundary_bitwise(oracle_mod, vsdmo):
    xyz, tri = square_with_boundary_jitter()
    om = oracle_mod.OracleMesh(TRI, xyz, tri)
    gm = vsdmo.DMOMeshTri(xyz, tri)
    opt = vsdmo.DMOTriFlatClass(gm, n_iter=4, fix_boundary=False)
    curves, fdeg, flags, sectors = opt.feature_state()
    assert sectors is None
    x = om.xyz
    fdeg_o, opt_o = om.feature_flags(x)
    vn = np.zeros_like(x); vn[:, 2] = 1
    curves_o = om.curves_f32(x, vn)
    assert np.array_equal(fdeg, fdeg_o) and np.array_equal(flags, opt_o) and flags.sum() > 20
    assert same_bits(curves, curves_o)
    state = dict(x0=x.copy(), nn=np.arange(len(x), dtype=np.int32), vn=vn, curves=curves_o, fdeg=fdeg_o, opt=opt_o)
    for it in range(4):
        x = _oracle_iteration(oracle_mod, om, x, state, True, None)
        opt.iterate(1)
        assert same_bits(gm.positions(), x), it
    # straight boundaries: the boundary vertices stay on their lines (up to the rounding of the
    # inverse-distance blend, exact on the lines through 0), corners stay put
    g = gm.positions(original_order=True)
    for i, p0 in enumerate(xyz):
        for a in range(2):
            if p0[a] == 0.0:
                assert g[i, a] == 0.0
            if p0[a] == 1.0:
                assert abs(g[i, a] - 1.0) < 1e-6
    moved = np.any(g != xyz, axis=1)
    bnd = np.array([(p[0] in (0.0, 1.0)) or (p[1] in (0.0, 1.0)) for p in xyz])
    assert moved[bnd].sum() > 10
    mn, mean = opt.history()
    assert np.all(np.diff(mn) >= -1e-6) and mean[-1] > mean[0]


@pytest.mark.parametrize("quads", [False, True])
def test_surface_with_features_bitwise(oracle_mod, vsdmo, quads):
    sx, faces = cube_surface_with_jitter(vsdmo, quads=quads)
    et = QUAD if quads else TRI
    om = oracle_mod.OracleMesh(et, sx, faces)
    gm = (vsdmo.DMOMeshQuad if quads else vsdmo.DMOMeshTri)(sx, faces)
    assert gm.info == om.info and gm.info["nFeature"] > 0
    opt = (vsdmo.DMOQuadClass if quads else vsdmo.DMOTriClass)(gm, n_iter=3)
    x0, ls, nn, fn, vn = om.surface_state_f32(om.xyz)
    sectors_o = om.sector_surfaces(om.xyz, fn)
    fdeg_o, opt_o = om.feature_flags(om.xyz)
    curves_o = om.curves_f32(om.xyz, vn)
    curves, fdeg, flags, sectors = opt.feature_state()
    assert np.array_equal(fdeg, fdeg_o) and np.array_equal(flags, opt_o) and flags.sum() > 0
    assert same_bits(curves, curves_o)
    assert np.array_equal(sectors[0], sectors_o[0]) and np.array_equal(sectors[1], sectors_o[1])
    assert same_bits(sectors[2], sectors_o[2])
    state = dict(x0=x0, ls=ls, nn=nn, vn=vn, fn=fn, curves=curves_o, fdeg=fdeg_o, opt=opt_o)
    x = om.xyz
    for it in range(3):
        x = _oracle_iteration(oracle_mod, om, x, state, False, sectors_o)
        opt.iterate(1)
        assert same_bits(gm.positions(), x), it
    # the cube: face vertices stay in their face plane, edge vertices on their edge
    g = gm.positions(original_order=True)
    for i, p0 in enumerate(sx):
        on = (np.abs(p0) < 1e-7) | (np.abs(p0 - 1) < 1e-7)
        assert np.all(np.abs(g[i, on] - p0[on]) < 1e-6), (i, p0, g[i])
    mn, mean = opt.history()
    assert np.all(np.diff(mn) >= -1e-6) and mean[-1] > mean[0]


def test_features_fixed_when_asked(vsdmo):
    sx, faces = cube_surface_with_jitter(vsdmo)
    gm = vsdmo.DMOMeshTri(sx, faces)
    nFree = gm.info["nSurf"] - gm.info["nFeature"]
    opt = vsdmo.DMOTriClass(gm, n_iter=2, fix_boundary=True)
    x = gm.positions()
    opt.optimize()
    g = gm.positions()
    assert np.array_equal(g[nFree:], x[nFree:]) and np.any(g[:nFree] != x[:nFree])


def test_flat_sliding_against_fp64_reference(oracle_mod, vsdmo):
    """One iteration (free classes, then the boundary pass) against the literal double
    restatement: positions within 1e-5 h wherever the double decisions are clear."""
    n = 16
    h = 1.0 / (n - 1)
    xyz, tri = square_with_boundary_jitter(n, seed=2)
    om = oracle_mod.OracleMesh(TRI, xyz, tri)
    gm = vsdmo.DMOMeshTri(xyz, tri)
    opt = vsdmo.DMOTriFlatClass(gm, n_iter=1, fix_boundary=False)
    x = om.xyz.astype(np.float64)
    clear = np.ones(len(x), bool)
    for (v0, v1) in om.color_ranges():
        x, mg = om.dmo_color_f64(x, v0, v1)
        clear[v0:v1] &= mg > 1e-5
    vn = np.zeros_like(x); vn[:, 2] = 1
    fdeg, flags = om.feature_flags(om.xyz)
    curves = om.curves_f64(om.xyz.astype(np.float64), vn)
    nn = np.arange(len(x), dtype=np.int32)
    cf = om.array(oracle_mod.A_COL_FEATURE)
    rp = om.array(oracle_mod.A_HE_ROWPTR)
    he = om.array(oracle_mod.A_HALFEDGES).reshape(-1, 4)
    for c in range(len(cf) - 1):
        v0, v1 = int(cf[c]), int(cf[c + 1])
        x, mg = om.dmo_1d_f64(x, om.xyz, curves, nn, vn, fdeg, flags, v0, v1)
        clear[v0:v1] &= mg > 1e-5
        # a boundary vertex sees the positions of its ring: it is comparable only when they are
        for v in range(v0, v1):
            clear[v] &= bool(np.all(clear[he[rp[v]:rp[v + 1], 0]]))
    opt.iterate(1)
    d = np.abs(gm.positions().astype(np.float64) - x).max(1)
    assert np.all(d[clear] < 1e-5 * h), float(d[clear].max())
    nFree = om.info["nSurf"] - om.info["nFeature"]
    assert clear[nFree:].sum() > 0.6 * (len(x) - nFree)


def test_flat_boundary_pass_waits_for_a_valid_mesh(oracle_mod, vsdmo):
    """DMOTriFlatClass runs the boundary pass only while the minimum quality is positive: with
    an inverted triangle at the start the boundary stays where it is in the first iteration."""
    xyz, tri = square_with_boundary_jitter(16, seed=5)
    om = oracle_mod.OracleMesh(TRI, xyz, tri)
    assert om.element_qualities_f32(om.xyz).min() < 0
    gm = vsdmo.DMOMeshTri(xyz, tri)
    opt = vsdmo.DMOTriFlatClass(gm, n_iter=1, fix_boundary=False, check_monotone=False)
    nFree = gm.info["nSurf"] - gm.info["nFeature"]
    x = gm.positions()
    opt.iterate(1)
    g = gm.positions()
    assert np.array_equal(g[nFree:], x[nFree:]) and np.any(g[:nFree] != x[:nFree])
