"""GPU tests of the flat 2D paths beyond the reference's triangle kernel: the general flat
search (4 or 8 candidates per axis, 1-4 levels, 8 / 16 / 32 lanes per vertex) on triangle and
quad meshes, single-mesh and batched (many meshes in one persistent launch per iteration),
bitwise against the oracle's f32 restatement (oracle/or_flat.c), the flat-quad search within
the FP64 tolerances of the literal restatement, and the batch's per-mesh statistics, graph
replay, autotuner and error reporting."""
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


def q_flat32(xyz, el):
    """Element qualities of flat tris / quads in float32 with the kernels' operation order."""
    p = xyz[el].astype(np.float32)
    if el.shape[1] == 3:
        e0, e1, e2 = p[:, 1] - p[:, 0], p[:, 2] - p[:, 1], p[:, 0] - p[:, 2]
        sq = lambda e: e[:, 0] * e[:, 0] + e[:, 1] * e[:, 1]
        l = (sq(e0) + sq(e1)) + sq(e2)
        area = e0[:, 0] * e1[:, 1] - e0[:, 1] * e1[:, 0]
        q = (np.float32(2.0) * np.sqrt(np.float32(3.0))) * area / l
        return np.where(area < 0, area, q).astype(np.float32)
    e0, e1, e2, e3 = p[:, 1] - p[:, 0], p[:, 2] - p[:, 1], p[:, 3] - p[:, 2], p[:, 0] - p[:, 3]
    sq = lambda e: e[:, 0] * e[:, 0] + e[:, 1] * e[:, 1]
    l = ((sq(e0) + sq(e1)) + sq(e2)) + sq(e3)
    c1 = e1[:, 0] * (-e0[:, 1]) - e1[:, 1] * (-e0[:, 0])
    c2 = e3[:, 0] * (-e2[:, 1]) - e3[:, 1] * (-e2[:, 0])
    q = (np.float32(2.0) * (c1 + c2)) / l
    return np.where((c1 < 0) | (c2 < 0), np.float32(-1.0), q).astype(np.float32)


def _to_original(om, x_internal):
    return x_internal[om.array(1)]   # new_of_old


def _oracle_iterations(oracle_mod, etype, xyz, el, iters, nq, depth, seed=1):
    om = oracle_mod.OracleMesh(etype, xyz, el, color_seed=seed)
    x = om.xyz
    for _ in range(iters):
        for (v0, v1) in om.color_ranges():
            x = om.dmo_flat_f32(x, v0, v1, nq=nq, depth=depth)
    return om, x


# ---- single mesh ---------------------------------------------------------------------------

@pytest.mark.parametrize("nq,depth", [(8, 3), (4, 2), (4, 4), (8, 1)])
def test_flat_quad_single_colour_bitwise(oracle_mod, vsdmo, nq, depth):
    xyz, el = G.quad_grid(24, seed=3, jitter=0.4)
    om = oracle_mod.OracleMesh(QUAD, xyz, el)
    gm = vsdmo.DMOMeshQuad(xyz, el)
    assert gm.info == om.info and gm.info["isFlat"] == 1
    opt = vsdmo.DMOQuadFlatClass(gm, n_iter=2, grid_n=nq, depth=depth)
    x = om.xyz
    moved = 0
    for c, (v0, v1) in enumerate(om.color_ranges()):
        y = om.dmo_flat_f32(x, v0, v1, nq=nq, depth=depth)
        moved += int(np.any(y != x, axis=1).sum())
        x = y
        opt.run_color(c)
        assert same_bits(gm.positions(), x), c
    assert moved > 0


def test_flat_tri_grid4_bitwise(oracle_mod, vsdmo):
    xyz, el = G.tri_grid(30, seed=5, jitter=0.4)
    om = oracle_mod.OracleMesh(TRI, xyz, el)
    gm = vsdmo.DMOMeshTri(xyz, el)
    opt = vsdmo.DMOTriFlatClass(gm, n_iter=3, grid_n=4, depth=4)
    opt.optimize()
    x = om.xyz
    for _ in range(3):
        for (v0, v1) in om.color_ranges():
            x = om.dmo_flat_f32(x, v0, v1, nq=4, depth=4)
    assert same_bits(gm.positions(), x)
    mn, _ = opt.history()
    assert np.all(np.diff(mn) >= -1e-6)


def test_flat_quad_full_run_and_stats(oracle_mod, vsdmo):
    xyz, el = G.quad_grid(40, seed=7, jitter=0.4)
    om, x = _oracle_iterations(oracle_mod, QUAD, xyz, el, 4, 8, 3)
    gm = vsdmo.DMOMeshQuad(xyz, el)
    opt = vsdmo.DMOQuadFlatClass(gm, n_iter=4)
    opt.optimize()
    assert same_bits(gm.positions(), x)
    q = opt.getElementQualities()
    qe = q_flat32(gm.positions(), gm.array(vsdmo.A_ELEMS).reshape(-1, 4))
    assert same_bits(q, qe)
    mn, mean = opt.history()
    assert np.all(np.diff(mn) >= -1e-6) and mean[-1] > mean[0]


def test_flat_quad_against_fp64_reference(oracle_mod, vsdmo):
    n = 40
    h = 1.0 / (n - 1)
    xyz, el = G.quad_grid(n, seed=9, jitter=0.4)
    om = oracle_mod.OracleMesh(QUAD, xyz, el)
    gm = vsdmo.DMOMeshQuad(xyz, el)
    opt = vsdmo.DMOQuadFlatClass(gm, n_iter=1)
    x = om.xyz
    checked = total = 0
    for c, (v0, v1) in enumerate(om.color_ranges()):
        x64, margin = om.dmo_quad2d_f64(x.astype(np.float64), v0, v1)
        opt.run_color(c)
        g = gm.positions()
        clear = margin > 1e-5
        d = np.abs(g[v0:v1].astype(np.float64) - x64[v0:v1]).max(1)
        assert np.all(d[clear] < 1e-5 * h), float(d[clear].max())
        checked += int(clear.sum())
        total += v1 - v0
        x = g
    # candidates that turn a corner clockwise all score -1: exact ties leave some vertices
    # without a decision margin
    assert checked > 0.8 * total


# ---- batched --------------------------------------------------------------------------------

def _small_batch():
    return [
        (TRI, *G.tri_grid(12, seed=11, jitter=0.4)),
        (QUAD, *G.quad_grid(15, seed=12, jitter=0.4)),
        (TRI, *G.tri_grid(33, seed=13, jitter=0.4)),
        (QUAD, *G.quad_grid(41, seed=14, jitter=0.4)),
        (TRI, *G.tri_grid(7, seed=15, jitter=0.4)),
        (QUAD, *G.quad_grid(23, seed=16, jitter=0.4)),
    ]


CONFIGS = [(8, 3, 32), (8, 3, 8), (4, 2, 16), (4, 4, 32), (8, 2, 16), (8, 4, 8)]


def test_batch_matches_per_mesh_oracle(oracle_mod, vsdmo):
    meshes = _small_batch()
    b = vsdmo.BatchDMO(meshes)
    info = b.info()
    assert info["meshes"] == len(meshes) and info["vertices"] == sum(len(p) for _, p, _ in meshes)
    nq = [c[0] for c in CONFIGS]
    dp = [c[1] for c in CONFIGS]
    ln = [c[2] for c in CONFIGS]
    b.set_config(nq, dp, ln)
    n, d, l = b.config()
    assert list(n) == nq and list(d) == dp and list(l) == ln
    b.iterate(3)
    pos = b.positions()
    off = 0
    for i, (t, xyz, el) in enumerate(meshes):
        om, x = _oracle_iterations(oracle_mod, t, xyz, el, 3, nq[i], dp[i])
        mi = b.mesh_info(i)
        assert mi["v_off"] == off and mi["nV"] == len(xyz) and mi["colors"] == len(om.color_ranges())
        got = pos[off:off + len(xyz)]
        assert same_bits(got, _to_original(om, x)), i
        off += len(xyz)


def test_batch_stats_and_monotone(oracle_mod, vsdmo):
    meshes = _small_batch()
    b = vsdmo.BatchDMO(meshes)
    b.iterate(4)
    mins = []
    for it in range(5):
        mn, mean, below = b.stats(it)
        mins.append(mn)
        if it > 0:
            assert np.all(below == 0)
    mins = np.array(mins)
    assert np.all(np.diff(mins, axis=0) >= -1e-6)
    pos = b.positions()
    mn, mean, _ = b.stats(4)
    off = 0
    for i, (t, xyz, el) in enumerate(meshes):
        q = q_flat32(pos[off:off + len(xyz)], el)
        assert mn[i] == q.min(), i
        assert abs(mean[i] - q.astype(np.float64).mean()) < 1e-6
        off += len(xyz)
    with pytest.raises(vsdmo.VSDMOError):
        b.stats(5)


def test_batch_async_restart_and_set_positions(oracle_mod, vsdmo):
    meshes = _small_batch()
    b1 = vsdmo.BatchDMO(meshes)
    b2 = vsdmo.BatchDMO(meshes)
    x0 = b1.positions()
    b1.iterate(2)
    b2.iterate_async(1)
    b2.iterate_async(1)
    b2.sync()
    assert same_bits(b1.positions(), b2.positions())
    # back to the start: the same two iterations again
    b1.set_positions(x0)
    b1.restart()
    assert b1.info()["iterations"] == 0
    b1.iterate(2)
    assert same_bits(b1.positions(), b2.positions())


def test_batch_autotune(oracle_mod, vsdmo):
    meshes = G.config4(seed=3, count=24, v_min=300, v_max=15000)
    b = vsdmo.BatchDMO(meshes)
    x0 = b.positions()
    rep = b.autotune(probe_iters=3)
    assert rep.count("bucket") >= 2, rep
    assert same_bits(b.positions(), x0)
    n, d, l = b.config()
    assert set(n) <= {4, 8} and set(d) <= {2, 3, 4} and set(l) <= {8, 16, 32}
    b.iterate(2)
    pos = b.positions()
    off = 0
    for i, (t, xyz, el) in enumerate(meshes):
        if i % 5 == 0:
            om, x = _oracle_iterations(oracle_mod, t, xyz, el, 2, int(n[i]), int(d[i]))
            assert same_bits(pos[off:off + len(xyz)], _to_original(om, x)), i
        off += len(xyz)


def test_batch_benchmark_workload(oracle_mod, vsdmo):
    meshes = G.config4()
    b = vsdmo.BatchDMO(meshes)
    assert b.info()["vertices"] == sum(len(p) for _, p, _ in meshes) == 3261948
    b.iterate(3)
    mins = np.array([b.stats(i)[0] for i in range(4)])
    assert np.all(np.diff(mins, axis=0) >= -1e-6)
    means = np.array([b.stats(i)[1] for i in range(4)])
    assert np.all(means[-1] > means[0])
    pos = b.positions()
    sizes = np.array([len(p) for _, p, _ in meshes])
    offs = np.concatenate([[0], np.cumsum(sizes)])
    for i in list(np.argsort(sizes)[:2]) + [int(np.argmax(sizes))]:
        t, xyz, el = meshes[i]
        om, x = _oracle_iterations(oracle_mod, t, xyz, el, 3, 8, 3)
        assert same_bits(pos[offs[i]:offs[i + 1]], _to_original(om, x)), i


def test_batch_argument_errors(vsdmo):
    meshes = _small_batch()
    b = vsdmo.BatchDMO(meshes)
    with pytest.raises(vsdmo.VSDMOError):
        b.set_config(5, 3, 32)
    with pytest.raises(vsdmo.VSDMOError):
        b.set_config(8, 5, 32)
    with pytest.raises(vsdmo.VSDMOError):
        b.set_config(8, 3, 12)
    # a mesh that is not flat
    xyz, el = G.tri_grid(8, seed=1)
    xyz = xyz.copy()
    xyz[5, 2] = 0.1
    with pytest.raises(vsdmo.VSDMOError):
        vsdmo.BatchDMO([(TRI, xyz, el)])
