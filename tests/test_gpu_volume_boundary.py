"""GPU parity tests of the boundary passes of volume meshes (DMOTetClass / DMOHexClass with a
free boundary, dmo/DMOTet.cu:128-170, dmo/DMOHex.cu:131-185): the interior classes, then —
while the minimum quality after the previous iteration is positive — the free boundary
classes on their local surfaces judged by their volume rings (k_optimizeHierarchical2DTet /
2DHex) and the feature classes on their curves (k_optimizeHierarchical1DTet / 1DHex), then the
nearest-initial-vertex walk and the normals. Bitwise against the oracle's f32 restatement over
whole iterations, within the FP64 restatement's tolerance for one iteration, and the known
answer of a cube: boundary vertices stay on their faces and edges."""
import ctypes as C

import numpy as np
import pytest

from volumesurfacediscretemeshoptimization_b200 import meshgen as G

pytestmark = pytest.mark.gpu
TET, HEX = 2, 3


def same_bits(a, b):
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape:
        return False
    na, nb = np.isnan(a), np.isnan(b)
    return bool(np.array_equal(na, nb) and np.array_equal(a[~na].view(np.uint32), b[~nb].view(np.uint32)))


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def jittered_cube(kind="tet", n=None, seed=4):
    """Tet (n = 6) or hex (n = 5) cube with interior vertices jittered by up to 0.3h (hex 0.2h)
    and boundary vertices displaced within their face plane / along their edge by up to 0.25h
    (hex 0.2h), corners fixed."""
    hex_ = kind == "hex"
    n = n or (5 if hex_ else 6)
    h = 1.0 / n
    ji, jb = (0.2, 0.2) if hex_ else (0.3, 0.25)
    xyz, el = (G.hex_cube if hex_ else G.tet_cube)(n, seed=None)
    xyz = xyz.astype(np.float64)
    rng = np.random.default_rng(seed)
    for i in range(len(xyz)):
        on = (np.abs(xyz[i]) < 1e-9) | (np.abs(xyz[i] - 1) < 1e-9)
        for a in range(3):
            if on.sum() == 0:
                xyz[i, a] += rng.uniform(-ji * h, ji * h)
            elif not on[a] and on.sum() < 3:
                xyz[i, a] += rng.uniform(-jb * h, jb * h)
    return xyz.astype(np.float32), el, h


def _classes(vsdmo, kind):
    return (HEX, vsdmo.DMOMeshHex, vsdmo.DMOHexClass) if kind == "hex" else (TET, vsdmo.DMOMeshTet, vsdmo.DMOTetClass)


def _ranges(arr):
    return [(int(arr[c]), int(arr[c + 1])) for c in range(len(arr) - 1)]


def _oracle_iteration(oracle_mod, om, x, st):
    """One DMOTetClass / DMOHexClass iteration with a free boundary on the oracle (f32)."""
    L = oracle_mod.lib()
    gate = om.element_qualities_f32(x).min() > 0
    for v0, v1 in _ranges(om.array(oracle_mod.A_COL_INNER)):
        x = om.dmo_color_f32(x, v0, v1)
    if gate:
        for v0, v1 in _ranges(om.array(oracle_mod.A_COL_FREE)):
            x = om.dmo_vol_surf_f32(x, st["x0"], st["ls"], st["nn"], st["sectors"], v0, v1)
        for v0, v1 in _ranges(om.array(oracle_mod.A_COL_FEATURE)):
            x = om.dmo_1d_f32(x, st["x0"], st["curves"], st["nn"], st["vn"], st["fdeg"], st["opt"], v0, v1)
    nn = st["nn"].copy()
    L.or_update_nn_f32(om.h, _p(np.ascontiguousarray(x, np.float32)), _p(st["x0"]), _p(nn))
    fn = np.zeros_like(st["fn"]); vn = np.zeros_like(st["vn"])
    L.or_surface_normals_f32(om.h, _p(np.ascontiguousarray(x, np.float32)), _p(fn), _p(vn))
    st.update(nn=nn, fn=fn, vn=vn)
    return x


@pytest.mark.parametrize("kind", ["tet", "hex"])
def test_free_boundary_bitwise(oracle_mod, vsdmo, kind):
    xyz, el, _ = jittered_cube(kind)
    et, Mesh, Opt = _classes(vsdmo, kind)
    om = oracle_mod.OracleMesh(et, xyz, el)
    gm = Mesh(xyz, el)
    assert gm.info == om.info and gm.info["nFeature"] > 0
    opt = Opt(gm, n_iter=3, fix_boundary=False)
    x = om.xyz
    x0, ls, nn, fn, vn = om.surface_state_f32(x)
    sectors_o = om.sector_surfaces(x, fn)
    fdeg_o, opt_o = om.feature_flags(x)
    curves_o = om.curves_f32(x, vn)
    # the optimiser's state: initial positions, local surfaces, curves, flags, sectors
    gx0, gls, gnn = opt.surface_state()
    assert same_bits(gx0, x[: len(gx0)]) and same_bits(gls, ls) and np.array_equal(gnn, nn)
    curves, fdeg, flags, sectors = opt.feature_state()
    assert np.array_equal(fdeg, fdeg_o) and np.array_equal(flags, opt_o) and flags.sum() > 0
    assert same_bits(curves, curves_o)
    assert np.array_equal(sectors[0], sectors_o[0]) and np.array_equal(sectors[1], sectors_o[1])
    assert same_bits(sectors[2], sectors_o[2])
    st = dict(x0=x0, ls=ls, nn=nn, fn=fn, vn=vn, sectors=sectors_o, curves=curves_o, fdeg=fdeg_o, opt=opt_o)
    for it in range(3):
        x = _oracle_iteration(oracle_mod, om, x, st)
        opt.iterate(1)
        assert same_bits(gm.positions(), x), it
    assert np.array_equal(opt.surface_state()[2], st["nn"])
    # the cube: face vertices stay in their face plane, edge vertices on their edge, and the
    # boundary moves
    g = gm.positions(original_order=True)
    nS = gm.info["nSurf"]
    on_bnd = np.zeros(len(xyz), bool)
    for i, p0 in enumerate(xyz):
        on = (np.abs(p0) < 1e-7) | (np.abs(p0 - 1) < 1e-7)
        on_bnd[i] = on.any()
        assert np.all(np.abs(g[i, on] - p0[on]) < 1e-6), (i, p0, g[i])
    assert on_bnd.sum() == nS
    assert np.any(g != xyz, axis=1)[on_bnd].sum() > nS // 2
    mn, mean = opt.history()
    assert np.all(np.diff(mn) >= -1e-6) and mean[-1] > mean[0]


@pytest.mark.parametrize("kind", ["tet", "hex"])
def test_free_boundary_against_fp64_reference(oracle_mod, vsdmo, kind):
    """The boundary passes of one iteration against the literal double restatement: from the
    positions after the interior classes (the f32 restatement's, bitwise the product's), the
    free boundary classes and the feature classes in double; positions within 1e-5 h wherever
    the double decisions are clear (a vertex is comparable when its own decisions and those of
    the boundary vertices of its volume ring are)."""
    xyz, el, h = jittered_cube(kind)
    et, Mesh, Opt = _classes(vsdmo, kind)
    om = oracle_mod.OracleMesh(et, xyz, el)
    gm = Mesh(xyz, el)
    opt = Opt(gm, n_iter=1, fix_boundary=False)
    x32 = om.xyz
    assert om.element_qualities_f64(x32.astype(np.float64)).min() > 0
    xi = x32
    for v0, v1 in _ranges(om.array(oracle_mod.A_COL_INNER)):
        xi = om.dmo_color_f32(xi, v0, v1)
    x = xi.astype(np.float64)
    nS = om.info["nSurf"]
    rp = om.array(oracle_mod.A_HF_ROWPTR)
    hf = om.array(oracle_mod.A_HALFFACES).reshape(-1, 7 if kind == "hex" else 3)
    clear = np.ones(len(x), bool)

    def ring_clear(v0, v1):
        for v in range(v0, v1):
            clear[v] &= bool(np.all(clear[hf[rp[v]:rp[v + 1]].ravel()]))

    x0, ls, nn, vn = om.surface_state_f64(x32)
    fn = om.array(oracle_mod.A_FACE_NORMALS).reshape(-1, 3).astype(np.float64)
    sectors = om.sector_surfaces(x32, fn, dtype=np.float64)
    for v0, v1 in _ranges(om.array(oracle_mod.A_COL_FREE)):
        x, mg = om.dmo_vol_surf_f64(x, x0, ls, nn, sectors, v0, v1)
        clear[v0:v1] &= mg > 1e-5
        ring_clear(v0, v1)
    fdeg, flags = om.feature_flags(x32)
    curves = om.curves_f64(x32, vn)
    for v0, v1 in _ranges(om.array(oracle_mod.A_COL_FEATURE)):
        x, mg = om.dmo_1d_f64(x, x0, curves, nn, vn, fdeg, flags, v0, v1)
        clear[v0:v1] &= mg > 1e-5
        ring_clear(v0, v1)
    opt.iterate(1)
    g = gm.positions()
    assert same_bits(g[nS:], xi[nS:])
    d = np.abs(g[:nS].astype(np.float64) - x[:nS]).max(1)
    c = clear[:nS]
    assert np.all(d[c] < 1e-5 * h), float(d[c].max())
    assert c.sum() > 0.5 * nS
    assert np.any(x[:nS] != x32[:nS])


@pytest.mark.parametrize("kind", ["tet", "hex"])
def test_boundary_fixed_by_default(vsdmo, kind):
    xyz, el, _ = jittered_cube(kind)
    _, Mesh, Opt = _classes(vsdmo, kind)
    gm = Mesh(xyz, el)
    nS = gm.info["nSurf"]
    x = gm.positions()
    Opt(gm, n_iter=2).optimize()
    g = gm.positions()
    assert np.array_equal(g[:nS], x[:nS]) and np.any(g[nS:] != x[nS:])


def test_tet_boundary_pass_waits_for_a_valid_mesh(oracle_mod, vsdmo):
    """With an inverted tet at the start the boundary stays where it is in the first iteration
    and the interior classes still move."""
    xyz, tets, _ = jittered_cube("tet")
    gm0 = vsdmo.DMOMeshTet(xyz, tets)
    nS = gm0.info["nSurf"]
    # push an interior vertex through a neighbouring boundary face
    inner = int(np.nonzero(np.all((xyz > 1e-6) & (xyz < 1 - 1e-6), axis=1))[0][0])
    bad = xyz.copy()
    bad[inner] = [bad[inner, 0], bad[inner, 1], -0.05]
    om = oracle_mod.OracleMesh(TET, bad, tets)
    assert om.element_qualities_f32(om.xyz).min() < 0
    gm = vsdmo.DMOMeshTet(bad, tets)
    opt = vsdmo.DMOTetClass(gm, n_iter=1, fix_boundary=False, check_monotone=False)
    x = gm.positions()
    opt.iterate(1)
    g = gm.positions()
    assert np.array_equal(g[:nS], x[:nS]) and np.any(g[nS:] != x[nS:])


def test_tet_free_boundary_with_active_set(vsdmo):
    """The active set skips only searches whose result cannot change: with the boundary passes
    (which move vertices of interior rings) the positions equal those of the full search."""
    xyz, tets, _ = jittered_cube("tet")
    out = []
    for active in (False, True):
        gm = vsdmo.DMOMeshTet(xyz, tets)
        vsdmo.DMOTetClass(gm, n_iter=6, fix_boundary=False, active_set=active).optimize()
        out.append(gm.positions())
    assert same_bits(out[0], out[1])
