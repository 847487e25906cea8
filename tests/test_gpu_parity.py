"""GPU parity tests: the CUDA library (through its C ABI) against the CPU oracle.

* connectivity and colouring: every array bit-exact (integers) / bitwise (float normals);
* grid search: bitwise equal to the oracle's restatement of the same float arithmetic, for
  single colour launches and whole multi-iteration runs;
* against the literal FP64 restatement of the reference kernels: positions within
  1e-5 * h wherever the FP64 decision margins are clear of rounding, and final minimum / mean
  element quality within 1e-4;
* full-size benchmark meshes: size-independent properties (monotone minimum quality, a
  bitwise-matching first colour launch, permutation round trip).
"""
import numpy as np
import pytest

from volumesurfacediscretemeshoptimization_b200 import meshgen as G

pytestmark = pytest.mark.gpu

MESHES = {
    "tri_grid8": (0, lambda: G.tri_grid(8, seed=3)),
    "config1": (0, lambda: G.config1()),
    "tri_grid_odd": (0, lambda: G.tri_grid(37, seed=11, jitter=0.45)),
    "icosphere3": (0, lambda: G.icosphere(3)),
    "tet_cube4": (2, lambda: G.tet_cube(4, seed=5)),
    "tet_cube12": (2, lambda: G.tet_cube(12, seed=0)),
    "tet_cube17": (2, lambda: G.tet_cube(17, seed=2, jitter=0.35)),
}


def same_bits(a, b):
    """Bitwise float equality; NaNs (e.g. the normal of a vertex whose face normals cancel)
    only need to sit at the same positions, since x86 and the GPU write different NaN bits."""
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape:
        return False
    na, nb = np.isnan(a), np.isnan(b)
    return bool(np.array_equal(na, nb) and np.array_equal(a[~na].view(np.uint32), b[~nb].view(np.uint32)))


def _pair(oracle_mod, vsdmo, name, seed=1):
    kind, gen = MESHES[name]
    xyz, el = gen()
    om = oracle_mod.OracleMesh(kind, xyz, el, color_seed=seed)
    gm = (vsdmo.DMOMeshTet if kind == 2 else vsdmo.DMOMeshTri)(xyz, el, color_seed=seed)
    return om, gm, xyz, el


@pytest.mark.parametrize("name", list(MESHES))
def test_connectivity_bit_exact(oracle_mod, vsdmo, name):
    om, gm, _, _ = _pair(oracle_mod, vsdmo, name)
    assert om.info == gm.info
    A, B = om.arrays(), gm.arrays()
    for k in A:
        a, b = A[k], B[k]
        assert a.shape == b.shape, k
        if a.dtype == np.float32:
            assert same_bits(a, b), k
        else:
            assert np.array_equal(a, b), k


def test_colour_seed_changes_colouring(oracle_mod, vsdmo):
    xyz, tets = G.tet_cube(6, seed=1)
    a = vsdmo.DMOMeshTet(xyz, tets, color_seed=1).array(vsdmo.A_COL_INNER)
    b = vsdmo.DMOMeshTet(xyz, tets, color_seed=2).array(vsdmo.A_COL_INNER)
    c = oracle_mod.OracleMesh(oracle_mod.TET, xyz, tets, color_seed=2).array(oracle_mod.A_COL_INNER)
    assert np.array_equal(b, c)
    assert not np.array_equal(a, b) or len(a) != len(b)


def test_permutation_round_trip(vsdmo):
    xyz, tets = G.tet_cube(5, seed=3)
    m = vsdmo.DMOMeshTet(xyz, tets)
    assert np.array_equal(m.positions(original_order=True), xyz)
    noo = m.permutation()
    assert np.array_equal(m.positions()[noo], xyz)
    y = xyz + 0.001
    m.set_positions(y, original_order=True)
    assert np.array_equal(m.positions(original_order=True), y.astype(np.float32))


def _opt(vsdmo, gm, **kw):
    cls = vsdmo.DMOTetClass if gm.elem_type == 2 else vsdmo.DMOTriFlatClass
    return cls(gm, **kw)


@pytest.mark.parametrize("name", ["tri_grid8", "config1", "tet_cube4", "tet_cube12"])
def test_single_colour_launches_bitwise(oracle_mod, vsdmo, name):
    om, gm, _, _ = _pair(oracle_mod, vsdmo, name)
    opt = _opt(vsdmo, gm, n_iter=1)
    x = om.xyz
    assert np.array_equal(gm.positions(), x)
    for c, (v0, v1) in enumerate(om.color_ranges()):
        x = om.dmo_color_f32(x, v0, v1)
        opt.run_color(c)
        g = gm.positions()
        assert np.array_equal(g.view(np.uint32), x.view(np.uint32)), (c, np.abs(g - x).max())


@pytest.mark.parametrize("name,iters", [("config1", 10), ("tri_grid_odd", 6), ("tet_cube12", 5), ("tet_cube17", 3)])
@pytest.mark.parametrize("use_graph", [True, False])
def test_full_runs_bitwise(oracle_mod, vsdmo, name, iters, use_graph):
    om, gm, _, _ = _pair(oracle_mod, vsdmo, name)
    opt = _opt(vsdmo, gm, n_iter=iters, use_graph=use_graph)
    x32, mn32, me32 = om.optimize_f32(om.xyz, iters)
    opt.optimize()
    assert opt.isDone()
    g = gm.positions()
    assert np.array_equal(g.view(np.uint32), x32.view(np.uint32))
    mn, mean = opt.history()
    assert len(mn) == iters + 1
    # the quality kernel uses CUDA cbrtf/sqrtf and a different summation order: 1e-6 level
    np.testing.assert_allclose(mn[1:], mn32, rtol=0, atol=2e-6)
    np.testing.assert_allclose(mean[1:], me32, rtol=0, atol=2e-6)
    assert np.all(np.diff(mn) >= -1e-6)


# Whole runs are held to 1e-4 while near-tie decisions have not compounded: on the 12^3 cube
# the float restatement of the search (bitwise equal to the library, test_full_runs_bitwise) is
# within 6e-5 of FP64 through iteration 4 and 1.1e-4 off in the mean at iteration 5; the
# full-size workloads have their own fixtures (test_gpu_full_size.py).
@pytest.mark.parametrize("name,iters,h", [("config1", 10, 1 / 63), ("tet_cube12", 4, 1 / 12)])
def test_against_fp64_reference(oracle_mod, vsdmo, name, iters, h):
    om, gm, _, _ = _pair(oracle_mod, vsdmo, name)
    opt = _opt(vsdmo, gm, n_iter=iters)
    # (1) per colour from identical state: positions within 1e-5 h where decisions are clear
    x = om.xyz
    checked = 0
    for c, (v0, v1) in enumerate(om.color_ranges()):
        x64, margin = om.dmo_color_f64(x.astype(np.float64), v0, v1)
        opt.run_color(c)
        g = gm.positions()
        clear = margin > 1e-5
        d = np.abs(g[v0:v1].astype(np.float64) - x64[v0:v1]).max(1)
        assert np.all(d[clear] < 1e-5 * h), float(d[clear].max())
        checked += int(clear.sum())
        x = g
    assert checked > 0.5 * sum(v1 - v0 for v0, v1 in om.color_ranges())
    # (2) whole run from the initial state: final min / mean quality within 1e-4
    gm2 = (vsdmo.DMOMeshTet if gm.elem_type == 2 else vsdmo.DMOMeshTri)(*MESHES[name][1]())
    opt2 = _opt(vsdmo, gm2, n_iter=iters)
    opt2.optimize()
    q_min, q_mean = opt2.quality_stats()
    _, mn64, me64 = om.optimize_f64(om.xyz, iters)
    assert abs(q_min - mn64[-1]) < 1e-4
    assert abs(q_mean - me64[-1]) < 1e-4


def test_element_quality_and_histogram(oracle_mod, vsdmo):
    om, gm, _, _ = _pair(oracle_mod, vsdmo, "tet_cube12")
    opt = _opt(vsdmo, gm, n_iter=2)
    q = opt.getElementQualities()
    q64 = om.element_qualities_f64(om.xyz)
    np.testing.assert_allclose(q, q64, rtol=0, atol=2e-6)
    hist = opt.getQualityHistogram(10)
    qq = np.minimum(q, 0.9999)
    ref = np.bincount(np.where(qq > 0, (qq * 10).astype(int), 0), minlength=10)
    assert np.array_equal(hist, ref)
    assert abs(opt.getQuality() - q.min()) < 1e-7


@pytest.mark.parametrize("cfg", ["config1", "config2"])
def test_benchmark_mesh_properties(oracle_mod, vsdmo, cfg):
    xyz, el = getattr(G, cfg)()
    kind = 0 if cfg == "config1" else 2
    gm = (vsdmo.DMOMeshTet if kind == 2 else vsdmo.DMOMeshTri)(xyz, el)
    om = oracle_mod.OracleMesh(kind, xyz, el)
    # connectivity of the full-size mesh, bit-exact
    for aid in (vsdmo.A_NEW_OF_OLD, vsdmo.A_COL_INNER, vsdmo.A_COL_FREE, vsdmo.A_HF_ROWPTR, vsdmo.A_HALFFACES,
                vsdmo.A_HE_ROWPTR, vsdmo.A_HALFEDGES, vsdmo.A_SURF_TRIS):
        assert np.array_equal(gm.array(aid), om.array(aid)), aid
    opt = _opt(vsdmo, gm, n_iter=10 if kind == 0 else 20)
    q0 = opt.getQuality()
    # first colour launch bitwise against the oracle on the full mesh
    (v0, v1) = om.color_ranges()[0]
    x = om.dmo_color_f32(om.xyz, v0, v1)
    opt.run_color(0)
    assert np.array_equal(gm.positions().view(np.uint32), x.view(np.uint32))
    opt.optimize()
    mn, mean = opt.history()
    assert np.all(np.diff(mn) >= -1e-6)
    assert mn[-1] > q0 and mn[-1] > 0
    assert mean[-1] > mean[0]
