"""GPU parity tests of the hexahedral path: hex connectivity (boundary quads, interior
colouring, the quad surface, halfhexes) bit-exact, and the interior grid search with the
reference's shape metric bitwise against the oracle's f32 restatement and within the FP64
tolerances of its literal restatement (oracle/or_hex.c)."""
import numpy as np
import pytest

from volumesurfacediscretemeshoptimization_b200 import meshgen as G

pytestmark = pytest.mark.gpu
HEX = 3

HEXES = {
    "hex3": lambda: G.hex_cube(3, seed=1),
    "hex5": lambda: G.hex_cube(5, seed=2),
    "hex8": lambda: G.hex_cube(8, seed=4),
    "hex7_clean": lambda: G.hex_cube(7, seed=None),
}


def same_bits(a, b):
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape:
        return False
    na, nb = np.isnan(a), np.isnan(b)
    return bool(np.array_equal(na, nb) and np.array_equal(a[~na].view(np.uint32), b[~nb].view(np.uint32)))


def _pair(oracle_mod, vsdmo, name, seed=1):
    xyz, el = HEXES[name]()
    om = oracle_mod.OracleMesh(HEX, xyz, el, color_seed=seed)
    gm = vsdmo.DMOMeshHex(xyz, el, color_seed=seed)
    return om, gm


@pytest.mark.parametrize("name", list(HEXES))
def test_hex_connectivity_bit_exact(oracle_mod, vsdmo, name):
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


@pytest.mark.parametrize("name", ["hex5", "hex8"])
def test_hex_single_colour_launches_bitwise(oracle_mod, vsdmo, name):
    om, gm = _pair(oracle_mod, vsdmo, name)
    opt = vsdmo.DMOHexClass(gm, n_iter=1)
    x = om.xyz
    moved = 0
    for c, (v0, v1) in enumerate(om.color_ranges()):
        y = om.dmo_color_f32(x, v0, v1)
        moved += int(np.any(y != x, axis=1).sum())
        x = y
        opt.run_color(c)
        assert same_bits(gm.positions(), x), c
    assert moved > 0


@pytest.mark.parametrize("use_graph", [True, False])
def test_hex_full_runs_bitwise(oracle_mod, vsdmo, use_graph):
    om, gm = _pair(oracle_mod, vsdmo, "hex8")
    opt = vsdmo.DMOHexClass(gm, n_iter=4, use_graph=use_graph)
    x32, mn32, me32 = om.optimize_f32(om.xyz, 4)
    opt.optimize()
    assert same_bits(gm.positions(), x32)
    mn, mean = opt.history()
    np.testing.assert_allclose(mn[1:], mn32, rtol=0, atol=2e-6)
    np.testing.assert_allclose(mean[1:], me32, rtol=0, atol=2e-6)
    assert np.all(np.diff(mn) >= -1e-6) and mean[-1] > mean[0]


def test_hex_unperturbed_is_a_fixed_point(oracle_mod, vsdmo):
    om, gm = _pair(oracle_mod, vsdmo, "hex7_clean")
    opt = vsdmo.DMOHexClass(gm, n_iter=2)
    q = opt.getElementQualities()
    assert np.all(np.abs(q - 1.0) < 1e-6)
    x = gm.positions()
    opt.optimize()
    assert np.array_equal(gm.positions(), x)


def test_hex_against_fp64_reference(oracle_mod, vsdmo):
    om, gm = _pair(oracle_mod, vsdmo, "hex8")
    h = 1.0 / 8
    opt = vsdmo.DMOHexClass(gm, n_iter=3)
    x = om.xyz
    checked = total = 0
    for c, (v0, v1) in enumerate(om.color_ranges()):
        x64, margin = om.dmo_color_f64(x.astype(np.float64), v0, v1)
        opt.run_color(c)
        g = gm.positions()
        clear = margin > 1e-5
        d = np.abs(g[v0:v1].astype(np.float64) - x64[v0:v1]).max(1)
        assert np.all(d[clear] < 1e-5 * h), float(d[clear].max())
        checked += int(clear.sum())
        total += v1 - v0
        x = g
    # exact ties in double (a ring minimum held by a constant sub-tet, or 0) are structural and
    # decide nothing; the remaining decisions are clear for most vertices
    assert checked > 0.6 * total
    xyz, el = HEXES["hex8"]()
    gm2 = vsdmo.DMOMeshHex(xyz, el)
    opt2 = vsdmo.DMOHexClass(gm2, n_iter=3)
    opt2.optimize()
    q_min, q_mean = opt2.quality_stats()
    _, mn64, me64 = om.optimize_f64(om.xyz, 3)
    assert abs(q_min - mn64[-1]) < 1e-4
    assert abs(q_mean - me64[-1]) < 1e-4


def test_hex_element_qualities(oracle_mod, vsdmo):
    om, gm = _pair(oracle_mod, vsdmo, "hex8")
    opt = vsdmo.DMOHexClass(gm, n_iter=2)
    opt.optimize()
    q = opt.getElementQualities()
    q64 = om.element_qualities_f64(gm.positions().astype(np.float64))
    np.testing.assert_allclose(q, q64, rtol=0, atol=2e-6)


def test_hex_benchmark_mesh_properties(oracle_mod, vsdmo):
    xyz, el = G.config2_hex()
    om = oracle_mod.OracleMesh(HEX, xyz, el)
    gm = vsdmo.DMOMeshHex(xyz, el)
    for aid in (vsdmo.A_NEW_OF_OLD, vsdmo.A_COL_INNER, vsdmo.A_HF_ROWPTR, vsdmo.A_HALFFACES, vsdmo.A_SURF_TRIS,
                vsdmo.A_COL_FREE, vsdmo.A_HALFEDGES):
        assert np.array_equal(gm.array(aid), om.array(aid)), aid
    opt = vsdmo.DMOHexClass(gm, n_iter=20)
    (v0, v1) = om.color_ranges()[0]
    x = om.dmo_color_f32(om.xyz, v0, v1)
    opt.run_color(0)
    assert same_bits(gm.positions(), x)
    opt.optimize()
    mn, mean = opt.history()
    # the reference's extent is the per-axis MINIMUM ring distance, tiny on a jittered lattice:
    # the mean quality rises, hexes with a degenerate corner can stay at 0
    assert np.all(np.diff(mn) >= -1e-6) and mean[-1] > mean[0]


# ---- condition-number quality (QualityCriterium.CONDITION, an addition) -------------------

def test_hex_condition_qualities(oracle_mod, vsdmo):
    """Element qualities: 1 on the unit cube, bitwise against the oracle's f32 restatement and
    within 1e-6 of its double one on a jittered cube (with inverted corners)."""
    for name in ("hex7_clean", "hex8"):
        om, gm = _pair(oracle_mod, vsdmo, name)
        opt = vsdmo.DMOHexClass(gm, qualityCriterium=vsdmo.QualityCriterium.CONDITION, n_iter=1)
        q = opt.getElementQualities()
        x = gm.positions()
        assert same_bits(q, om.hex_cond_qualities(x, np.float32))
        np.testing.assert_allclose(q, om.hex_cond_qualities(x.astype(np.float64)), rtol=0, atol=1e-6)
        if name == "hex7_clean":
            assert np.all(np.abs(q - 1.0) < 1e-6)
        else:
            assert q.min() < 0


@pytest.mark.parametrize("name", ["hex3", "hex5", "hex8"])
def test_hex_condition_colour_launches_bitwise(oracle_mod, vsdmo, name):
    om, gm = _pair(oracle_mod, vsdmo, name)
    opt = vsdmo.DMOHexClass(gm, qualityCriterium=vsdmo.QualityCriterium.CONDITION, n_iter=2)
    x = om.xyz
    moved = 0
    for sweep in range(2):
        for c, (v0, v1) in enumerate(om.color_ranges()):
            y = om.dmo_hex_cond_f32(x, v0, v1)
            moved += int(np.any(y != x, axis=1).sum())
            x = y
            opt.run_color(c)
            assert same_bits(gm.positions(), x), (sweep, c)
    assert moved > 0


def test_hex_condition_against_fp64_and_known_answers(oracle_mod, vsdmo):
    """Colour launches within 1e-5 h of the literal double search where its decisions are
    clear (exact ties of constant corners decide nothing); a full run raises the minimum from
    inverted to valid monotonically; the unit-cube grid is a fixed point."""
    om, gm = _pair(oracle_mod, vsdmo, "hex8")
    h = 1.0 / 8
    opt = vsdmo.DMOHexClass(gm, qualityCriterium=vsdmo.QualityCriterium.CONDITION, n_iter=4)
    x = om.xyz
    checked = total = 0
    for c, (v0, v1) in enumerate(om.color_ranges()):
        x64, margin = om.dmo_hex_cond_f64(x.astype(np.float64), v0, v1)
        opt.run_color(c)
        g = gm.positions()
        clear = margin > 1e-5
        d = np.abs(g[v0:v1].astype(np.float64) - x64[v0:v1]).max(1)
        assert np.all(d[clear] < 1e-5 * h), float(d[clear].max())
        checked += int(clear.sum())
        total += v1 - v0
        x = g
    assert checked > 0.6 * total
    xyz, el = HEXES["hex8"]()
    opt2 = vsdmo.DMOHexClass(vsdmo.DMOMeshHex(xyz, el), qualityCriterium=vsdmo.QualityCriterium.CONDITION, n_iter=4,
                             check_monotone=False)
    q0 = opt2.getQuality()
    opt2.optimize()
    mn, mean = opt2.history()
    assert q0 < 0 < mn[-1] and np.all(np.diff(mn) >= -1e-6) and mean[-1] > mean[0]
    xyz, el = HEXES["hex7_clean"]()
    gm3 = vsdmo.DMOMeshHex(xyz, el)
    x3 = gm3.positions()
    vsdmo.DMOHexClass(gm3, qualityCriterium=vsdmo.QualityCriterium.CONDITION, n_iter=2).optimize()
    assert np.array_equal(gm3.positions(), x3)


def test_hex_condition_requires_fixed_boundary(vsdmo):
    xyz, el = HEXES["hex3"]()
    with pytest.raises(vsdmo.VSDMOError):
        vsdmo.DMOHexClass(vsdmo.DMOMeshHex(xyz, el), qualityCriterium=vsdmo.QualityCriterium.CONDITION,
                          fix_boundary=False)
    xyz, el = G.tet_cube(3, seed=1)
    with pytest.raises(vsdmo.VSDMOError):
        vsdmo.DMOTetClass(vsdmo.DMOMeshTet(xyz, el), qualityCriterium=vsdmo.QualityCriterium.CONDITION)
