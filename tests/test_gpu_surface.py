"""GPU parity tests of the surface path (tri and quad surface meshes without feature vertices).

Through the C ABI against the CPU oracle (oracle/or_surf.c, oracle/or_conn.c):
* quad connectivity and colouring bit-exact;
* the optimiser's initial state (initial positions, local quadric surfaces, nearest
  neighbours) bitwise;
* single colour launches and whole multi-iteration runs (grid search, nearest-neighbour walk,
  normal update) bitwise against the oracle's f32 restatement;
* against the literal FP64 restatement: positions within 1e-5 h where the FP64 decision
  margins are clear of rounding, final minimum / mean quality within 1e-4;
* the full-size surface workloads (icosphere level 7, torus 512 x 256): connectivity
  bit-exact, first colour launch bitwise, monotone minimum quality.
"""
import numpy as np
import pytest

from volumesurfacediscretemeshoptimization_b200 import meshgen as G

pytestmark = pytest.mark.gpu

TRI, QUAD = 0, 1


def _ico(level, seed, t):
    v, f = G.icosphere(level)
    return G.perturb_surface(v, f, seed=seed, tangential=t), f


def _torus(nu, nv, seed, t):
    v, q = G.torus_quads(nu, nv)
    return G.perturb_surface(v, q, seed=seed, tangential=t), q


SURF = {
    "ico3": (TRI, lambda: _ico(3, 1, 0.3), 0.15),
    "ico4": (TRI, lambda: _ico(4, 2, 0.3), 0.075),
    "ico3_clean": (TRI, lambda: G.icosphere(3), 0.15),
    "torus64x32": (QUAD, lambda: _torus(64, 32, 1, 0.2), 0.1),
    "torus40x40": (QUAD, lambda: _torus(40, 40, 2, 0.15), 0.15),
}


def same_bits(a, b):
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape:
        return False
    na, nb = np.isnan(a), np.isnan(b)
    return bool(np.array_equal(na, nb) and np.array_equal(a[~na].view(np.uint32), b[~nb].view(np.uint32)))


def _pair(oracle_mod, vsdmo, name, seed=1):
    kind, gen, _ = SURF[name]
    xyz, el = gen()
    om = oracle_mod.OracleMesh(kind, xyz, el, color_seed=seed)
    assert om.info["nFeature"] == 0, "test meshes must be free of feature vertices"
    gm = (vsdmo.DMOMeshQuad if kind == QUAD else vsdmo.DMOMeshTri)(xyz, el, color_seed=seed)
    return om, gm


def _opt(vsdmo, gm, **kw):
    cls = vsdmo.DMOQuadClass if gm.elem_type == QUAD else vsdmo.DMOTriClass
    return cls(gm, **kw)


@pytest.mark.parametrize("name", list(SURF))
def test_surface_connectivity_bit_exact(oracle_mod, vsdmo, name):
    om, gm = _pair(oracle_mod, vsdmo, name)
    assert om.info == gm.info
    A, B = om.arrays(), gm.arrays()
    for k in A:
        a, b = A[k], B[k]
        assert a.shape == b.shape, k
        if a.dtype == np.float32:
            assert same_bits(a, b), k
        else:
            assert np.array_equal(a, b), k


@pytest.mark.parametrize("name", list(SURF))
def test_surface_state_bitwise(oracle_mod, vsdmo, name):
    om, gm = _pair(oracle_mod, vsdmo, name)
    opt = _opt(vsdmo, gm, n_iter=1)
    x0, ls, nn = opt.surface_state()
    ox0, ols, onn, _, _ = om.surface_state_f32(om.xyz)
    assert same_bits(x0, ox0)
    assert same_bits(ls, ols), np.argwhere(ls.view(np.uint32) != ols.view(np.uint32))[:5]
    assert np.array_equal(nn, onn)
    # valence-4 vertices (quads) use the midpoint: 6 points; triangles: 1 + valence
    npts = ls[:, 15]
    assert np.all(npts >= 6)


@pytest.mark.parametrize("name", list(SURF))
def test_surface_single_colour_launches_bitwise(oracle_mod, vsdmo, name):
    om, gm = _pair(oracle_mod, vsdmo, name)
    opt = _opt(vsdmo, gm, n_iter=1)
    state = om.surface_state_f32(om.xyz)
    x = om.xyz
    moved = 0
    for c, (v0, v1) in enumerate(om.color_ranges()):
        y = om.dmo_surf_color_f32(x, state, v0, v1)
        moved += int(np.any(y != x, axis=1).sum())
        x = y
        opt.run_color(c)
        g = gm.positions()
        assert same_bits(g, x), (c, float(np.abs(g - x).max()))
    assert moved > 0


@pytest.mark.parametrize("name,iters", [("ico3", 6), ("ico4", 4), ("torus64x32", 4), ("torus40x40", 5)])
@pytest.mark.parametrize("use_graph", [True, False])
def test_surface_full_runs_bitwise(oracle_mod, vsdmo, name, iters, use_graph):
    om, gm = _pair(oracle_mod, vsdmo, name)
    opt = _opt(vsdmo, gm, n_iter=iters, use_graph=use_graph)
    x32, mn32, me32 = om.optimize_f32(om.xyz, iters)
    opt.optimize()
    assert opt.isDone()
    assert same_bits(gm.positions(), x32)
    _, _, nn = opt.surface_state()
    assert nn.min() >= 0 and nn.max() < om.info["nSurf"]
    mn, mean = opt.history()
    assert len(mn) == iters + 1
    np.testing.assert_allclose(mn[1:], mn32, rtol=0, atol=2e-6)
    np.testing.assert_allclose(mean[1:], me32, rtol=0, atol=2e-6)
    assert np.all(np.diff(mn) >= -1e-6)
    assert mean[-1] > mean[0]


@pytest.mark.parametrize("name,iters", [("ico3", 5), ("ico4", 3), ("torus64x32", 3)])
def test_surface_against_fp64_reference(oracle_mod, vsdmo, name, iters):
    h = SURF[name][2]
    om, gm = _pair(oracle_mod, vsdmo, name)
    opt = _opt(vsdmo, gm, n_iter=iters)
    # (1) one iteration colour by colour from the same state: positions within 1e-5 h where
    #     every FP64 decision of the vertex is clear of rounding
    x0, ls, nn, vn = om.surface_state_f64(om.xyz)
    x = om.xyz.astype(np.float64)
    checked = total = 0
    for c, (v0, v1) in enumerate(om.color_ranges()):
        x64, margin = om.dmo_surf_color_f64(x, x0, ls, nn, vn, v0, v1)
        opt.run_color(c)
        g = gm.positions()
        clear = margin > 1e-5
        d = np.abs(g[v0:v1].astype(np.float64) - x64[v0:v1]).max(1)
        assert np.all(d[clear] < 1e-5 * h), float(d[clear].max())
        checked += int(clear.sum())
        total += v1 - v0
        x = g.astype(np.float64)
    assert checked > 0.5 * total
    # (2) whole runs: final min / mean quality within 1e-4
    kind, gen, _ = SURF[name]
    xyz, el = gen()
    gm2 = (vsdmo.DMOMeshQuad if kind == QUAD else vsdmo.DMOMeshTri)(xyz, el)
    opt2 = _opt(vsdmo, gm2, n_iter=iters)
    opt2.optimize()
    q_min, q_mean = opt2.quality_stats()
    _, mn64, me64 = om.optimize_f64(om.xyz, iters)
    assert abs(q_min - mn64[-1]) < 1e-4
    assert abs(q_mean - me64[-1]) < 1e-4


def test_surface_element_qualities(oracle_mod, vsdmo):
    for name in ("ico3", "torus64x32"):
        om, gm = _pair(oracle_mod, vsdmo, name)
        opt = _opt(vsdmo, gm, n_iter=2)
        opt.optimize()
        q = opt.getElementQualities()
        q64 = om.element_qualities_f64(gm.positions().astype(np.float64))
        np.testing.assert_allclose(q, q64, rtol=0, atol=2e-6)
        assert abs(opt.getQuality() - q.min()) < 1e-7


def test_surface_meshes_with_features_are_accepted(vsdmo):
    # a coarse torus: 30 degrees between neighbouring quads around the tube -> all feature
    v, q = G.torus_quads(24, 12)
    gm = vsdmo.DMOMeshQuad(v, q)
    assert gm.info["nFeature"] > 0
    opt = vsdmo.DMOQuadClass(gm, n_iter=2)
    opt.optimize()
    mn, _ = opt.history()
    assert np.all(np.diff(mn) >= -1e-6)


def test_surface_restart_rebuilds_state(oracle_mod, vsdmo):
    om, gm = _pair(oracle_mod, vsdmo, "ico3")
    opt = _opt(vsdmo, gm, n_iter=3)
    x_init = gm.positions()
    opt.optimize()
    first = gm.positions()
    gm.set_positions(x_init)
    opt.restart()
    x0, ls, nn = opt.surface_state()
    assert same_bits(x0, x_init) and np.array_equal(nn, np.arange(len(nn)))
    opt.optimize()
    assert same_bits(gm.positions(), first)


@pytest.mark.parametrize("cfg", ["config3_tri", "config3_quad"])
def test_surface_restart_with_features_replays_bitwise(vsdmo, cfg):
    """restart() rebuilds the feature state; from the same positions the movable feature
    vertices and the sector surfaces come out the same, and the captured iterations are kept
    (they are dropped when either changes). The second run repeats the first bit for bit, and
    a restart from other positions matches a fresh optimiser started there."""
    xyz, el = getattr(G, cfg)()
    tri = cfg.endswith("tri")
    mcls, ocls = (vsdmo.DMOMeshTri, vsdmo.DMOTriClass) if tri else (vsdmo.DMOMeshQuad, vsdmo.DMOQuadClass)
    m = mcls(xyz, el)
    assert m.info["nFeature"] > 0
    o = ocls(m, n_iter=3)
    x0 = m.positions()
    o.optimize()
    first, h1 = m.positions(), o.history()
    m.set_positions(x0)
    o.restart()
    o.optimize()
    assert same_bits(m.positions(), first)
    assert np.array_equal(np.asarray(o.history()), np.asarray(h1))
    m.set_positions(first)
    o.restart()
    o.optimize()
    m2 = mcls(xyz, el)
    m2.set_positions(first)
    o2 = ocls(m2, n_iter=3)
    o2.optimize()
    assert same_bits(m.positions(), m2.positions())


@pytest.mark.parametrize("cfg,kind,iters", [("config3_tri", TRI, 15), ("config3_quad", QUAD, 15)])
def test_surface_benchmark_mesh_properties(oracle_mod, vsdmo, cfg, kind, iters):
    """the feature-free variant of the config 3 meshes (the specified noise is covered by
    test_gpu_full_size.py)"""
    xyz, el = getattr(G, cfg)(variant="feature_free")
    om = oracle_mod.OracleMesh(kind, xyz, el)
    assert om.info["nFeature"] == 0
    gm = (vsdmo.DMOMeshQuad if kind == QUAD else vsdmo.DMOMeshTri)(xyz, el)
    for aid in (vsdmo.A_NEW_OF_OLD, vsdmo.A_COL_FREE, vsdmo.A_HE_ROWPTR, vsdmo.A_HALFEDGES, vsdmo.A_SURF_TRIS):
        assert np.array_equal(gm.array(aid), om.array(aid)), aid
    opt = _opt(vsdmo, gm, n_iter=iters)
    state = om.surface_state_f32(om.xyz)
    _, ls, _ = opt.surface_state()
    assert same_bits(ls, state[1])
    (v0, v1) = om.color_ranges()[0]
    x = om.dmo_surf_color_f32(om.xyz, state, v0, v1, nthreads=0)
    opt.run_color(0)
    assert same_bits(gm.positions(), x)
    opt.optimize()
    mn, mean = opt.history()
    assert np.all(np.diff(mn) >= -1e-6)
    assert mean[-1] > mean[0]


@pytest.mark.parametrize("name", ["ico3", "torus64x32"])
def test_surface_view_samples_bitwise(oracle_mod, vsdmo, name):
    """getLocalSurfacePoints / getEstimateLocalSurfacePoints: the sample grids of the GUI's
    surface views, after two iterations (moved vertices, walked nearest neighbours), bitwise
    against the oracle with the optimiser's own state."""
    om, gm = _pair(oracle_mod, vsdmo, name)
    opt = _opt(vsdmo, gm, n_iter=2)
    opt.optimize()
    state = opt.surface_state()
    x = gm.positions()
    for vid in (0, 7, gm.info["nSurf"] - 1):
        for est, fn in ((False, opt.getLocalSurfacePoints), (True, opt.getEstimateLocalSurfacePoints)):
            g = fn(vid, 5, 7)
            o = om.surface_points_f32(x, state, vid, 5, 7, est)
            assert g.shape == (35, 3) and np.all(np.isfinite(g))
            assert same_bits(g, o), (vid, est)
    with pytest.raises(vsdmo.VSDMOError):
        opt.getLocalSurfacePoints(gm.info["nSurf"], 4, 4)


@pytest.mark.parametrize("name", ["ico3", "torus40x40"])
def test_two_ring_fit_bitwise(oracle_mod, vsdmo, name):
    """fit_ring=2 (an addition: the reference fits over the 1-ring): the quadrics over the
    2-ring bitwise against the oracle (or_surface_fit_ring_f32), within 1e-4 (relative) of its
    double fit, and colour launches on them bitwise."""
    om, gm = _pair(oracle_mod, vsdmo, name)
    opt = _opt(vsdmo, gm, n_iter=1, fit_ring=2)
    _, ls, _ = opt.surface_state()
    state = om.surface_state_f32(om.xyz, ring=2)
    assert same_bits(ls, state[1])
    # triangles: 1 + 6 + 12 points around a valence-6 vertex; quads: 1 + 4 + 8 (no midpoint)
    npts = ls[:, 15]
    assert npts.min() >= (13 if gm.elem_type == QUAD else 16)
    ls64 = om.surface_state_f64(om.xyz, ring=2)[1]
    # the 3 x 3 normal equations in float: relative error ~1e-5 of the coefficients
    np.testing.assert_allclose(ls[:, [3, 7, 11]], ls64[:, [3, 7, 11]], rtol=1e-4, atol=1e-5)
    ls1 = om.surface_state_f32(om.xyz, ring=1)[1]
    assert not same_bits(ls, ls1)
    x = om.xyz
    for c, (v0, v1) in enumerate(om.color_ranges()):
        x = om.dmo_surf_color_f32(x, state, v0, v1)
        opt.run_color(c)
        assert same_bits(gm.positions(), x), c


def test_two_ring_fit_on_a_sphere(oracle_mod, vsdmo):
    """Known answer: on the unit icosphere the quadric w = a u^2 + b uv + c v^2 of the sphere
    around a vertex has a = c = -1/2, b = 0 (w along the outward normal); both fits find it
    within the icosphere's chord error."""
    xyz, f = G.icosphere(4)
    for ring in (1, 2):
        gm = vsdmo.DMOMeshTri(xyz, f)
        opt = vsdmo.DMOTriClass(gm, n_iter=1, fit_ring=ring)
        ls = opt.surface_state()[1]
        assert np.all(np.abs(ls[:, 3] + 0.5) < 0.03) and np.all(np.abs(ls[:, 11] + 0.5) < 0.03)
        assert np.all(np.abs(ls[:, 7]) < 0.03)


@pytest.mark.parametrize("name", ["torus64x32", "torus40x40"])
def test_quad_condition_bitwise(oracle_mod, vsdmo, name):
    """QualityCriterium.CONDITION on quad surfaces (an addition: per corner 2 det / (|e1|^2 +
    |e2|^2), det signed by the vertex normal in the search): element qualities, single colour
    launches and whole runs bitwise against the oracle's f32 restatement under
    oracle.criterion(CONDITION)."""
    om, gm = _pair(oracle_mod, vsdmo, name)
    cond = vsdmo.QualityCriterium.CONDITION
    with oracle_mod.criterion(oracle_mod.CONDITION):
        opt = _opt(vsdmo, gm, qualityCriterium=cond, n_iter=1)
        assert same_bits(opt.getElementQualities(), om.element_qualities_f32(om.xyz))
        state = om.surface_state_f32(om.xyz)
        x = om.xyz
        for c, (v0, v1) in enumerate(om.color_ranges()):
            x = om.dmo_surf_color_f32(x, state, v0, v1)
            opt.run_color(c)
            assert same_bits(gm.positions(), x), c
        om2, gm2 = _pair(oracle_mod, vsdmo, name)
        opt2 = _opt(vsdmo, gm2, qualityCriterium=cond, n_iter=3)
        x32, mn32, me32 = om2.optimize_f32(om2.xyz, 3)
        opt2.optimize()
        assert same_bits(gm2.positions(), x32)
        mn, mean = opt2.history()
        np.testing.assert_allclose(mn[1:], mn32, rtol=0, atol=2e-6)
        assert np.all(np.diff(mn) >= -1e-6) and mean[-1] > mean[0]


def test_quad_condition_against_fp64_and_known_answers(oracle_mod, vsdmo):
    om, gm = _pair(oracle_mod, vsdmo, "torus64x32")
    h = SURF["torus64x32"][2]
    cond = vsdmo.QualityCriterium.CONDITION
    opt = _opt(vsdmo, gm, qualityCriterium=cond, n_iter=1)
    with oracle_mod.criterion(oracle_mod.CONDITION):
        np.testing.assert_allclose(opt.getElementQualities(), om.element_qualities_f64(om.xyz.astype(np.float64)),
                                   rtol=0, atol=1e-6)
        x0, ls, nn, vn = om.surface_state_f64(om.xyz)
        x = om.xyz
        checked = total = 0
        for c, (v0, v1) in enumerate(om.color_ranges()):
            x64, margin = om.dmo_surf_color_f64(x.astype(np.float64), x0, ls, nn, vn, v0, v1)
            opt.run_color(c)
            g = gm.positions()
            clear = margin > 1e-5
            d = np.abs(g[v0:v1].astype(np.float64) - x64[v0:v1]).max(1)
            assert np.all(d[clear] < 1e-5 * h), float(d[clear].max())
            checked += int(clear.sum())
            total += v1 - v0
            x = g
    assert checked > 0.5 * total
    # a square grid treated as a surface: every corner is square (quality 1), a fixed point
    xyz, q = G.quad_grid(12, seed=None)
    gq = vsdmo.DMOMeshQuad(xyz, q)
    oq = vsdmo.DMOQuadClass(gq, qualityCriterium=cond, n_iter=2)
    assert np.all(np.abs(oq.getElementQualities() - 1.0) < 1e-6)
    x = gq.positions()
    oq.optimize()
    assert np.array_equal(gq.positions(), x)
    # flat quad meshes (the 2D search) keep the mean ratio only
    with pytest.raises(vsdmo.VSDMOError):
        vsdmo.DMOQuadFlatClass(vsdmo.DMOMeshQuad(xyz, q), qualityCriterium=cond)
