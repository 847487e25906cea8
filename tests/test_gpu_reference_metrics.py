"""The oracle's metric restatements and the library's element qualities against the reference's
own quality functions: dmo/DMOQuality.h of the reference, compiled as it lies into
oracle/_ref/libref_quality.so (oracle/Makefile target ``ref``, oracle/ref_quality.cu) and
evaluated on the GPU.

Same elements, same criterion on every side. The reference computes in FP32 (its own build
flags: nvcc defaults, FMA contraction on), the oracle's restatements in FP64 and the library in
FP32. Tolerances: mean ratio and shape metric within 2e-6 absolute plus 1e-5 relative (the
inverted-element branches return a signed volume or area, not a bounded quality); angle
metrics within 2e-5 (CUDA's acosf against the FP64 acos)."""
import numpy as np
import pytest

from volumesurfacediscretemeshoptimization_b200 import meshgen as G

pytestmark = pytest.mark.gpu
MR_TOL = dict(rtol=1e-5, atol=2e-6)
ANGLE_TOL = dict(rtol=0, atol=2e-5)
# the unit cube in the reference's hex corner order (top face first, as meshgen.hex_cube writes it)
HEX_UNIT = np.array([[0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1], [0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], float)


@pytest.fixture(scope="module")
def ref(oracle_mod):
    if oracle_mod.ref_lib() is None:
        pytest.skip("the reference's quality functions were not built (its sources were absent at build time)")
    return oracle_mod


def _assert_close(a, b, tol):
    """Within tol where the value is a quality; the inverted-element branch (negative) returns
    a signed volume or area computed from absolute FP32 coordinates, whose cancellation leaves
    a relative error of order 1e-5, so it gets a relative bound."""
    neg = b < 0
    np.testing.assert_allclose(a[~neg], b[~neg], **tol)
    np.testing.assert_allclose(a[neg], b[neg], rtol=2e-4, atol=tol["atol"])


def _crits(R):
    return [R.REF_MEAN_RATIO, R.REF_MIN_ANGLE, R.REF_MAX_ANGLE]


def _tol(R, crit):
    return MR_TOL if crit == R.REF_MEAN_RATIO else ANGLE_TOL


def _lib_crit(vsdmo, R, crit):
    return {R.REF_MEAN_RATIO: vsdmo.QualityCriterium.MEAN_RATIO, R.REF_MIN_ANGLE: vsdmo.QualityCriterium.MIN_ANGLE,
            R.REF_MAX_ANGLE: vsdmo.QualityCriterium.MAX_ANGLE}[crit]


def _random_elements(rng, n, k, spread):
    """n elements of k corners: a jittered regular shape (spread < 1 keeps most valid; larger
    spreads fold many of them)."""
    base = {3: np.array([[0, 0, 0], [1, 0, 0], [0.5, np.sqrt(3) / 2, 0]]),
            4: np.array([[0, 0, 0], [1, 0, 0], [0.5, np.sqrt(3) / 2, 0], [0.5, np.sqrt(3) / 6, np.sqrt(2 / 3)]]),
            8: HEX_UNIT}[k]
    scale = rng.uniform(0.01, 10.0, size=(n, 1, 1))
    shift = rng.uniform(-5, 5, size=(n, 1, 3))
    return (base[None] + rng.uniform(-spread, spread, size=(n, k, 3))) * scale + shift


def test_known_answers(ref):
    R = ref
    tet = np.array([[[0, 0, 0], [1, 0, 0], [0.5, np.sqrt(3) / 2, 0], [0.5, np.sqrt(3) / 6, np.sqrt(2 / 3)]]])
    cube = HEX_UNIT[None]
    tri = np.array([[[0, 0, 0], [1, 0, 0], [0.5, np.sqrt(3) / 2, 0]]])
    assert abs(R.ref_quality(R.RQ_TET, R.REF_MEAN_RATIO, tet)[0] - 1) < 1e-6
    assert abs(R.ref_quality(R.RQ_HEX, R.REF_MEAN_RATIO, cube)[0] - 1) < 1e-6
    assert abs(R.ref_quality(R.RQ_TRI2D, R.REF_MEAN_RATIO, tri)[0] - 1) < 1e-6
    # a flipped element returns its signed volume / area (negative)
    assert R.ref_quality(R.RQ_TET, R.REF_MEAN_RATIO, tet[:, [1, 0, 2, 3]])[0] < 0
    assert R.ref_quality(R.RQ_TRI2D, R.REF_MEAN_RATIO, tri[:, [1, 0, 2]])[0] < 0


@pytest.mark.parametrize("spread", [0.3, 1.0])
def test_oracle_tet_metrics_match_reference(ref, spread):
    R = ref
    pts = _random_elements(np.random.default_rng(11), 3000, 4, spread)
    for crit in _crits(R):
        q_ref = R.ref_quality(R.RQ_TET, crit, pts)
        q64 = R.element_metric_f64(R.RQ_TET, crit, pts.astype(np.float32))
        if crit != R.REF_MEAN_RATIO:
            # an angle's sensitivity to rounding grows without bound as the element flattens
            keep = np.abs(R.element_metric_f64(R.RQ_TET, R.REF_MEAN_RATIO, pts.astype(np.float32))) > 0.05
            q_ref, q64 = q_ref[keep], q64[keep]
        _assert_close(q_ref, q64, _tol(R, crit))
    if spread >= 1.0:
        assert (R.ref_quality(R.RQ_TET, R.REF_MEAN_RATIO, pts) < 0).mean() > 0.1


@pytest.mark.parametrize("spread", [0.2, 0.6])
def test_oracle_hex_metric_matches_reference(ref, spread):
    R = ref
    pts = _random_elements(np.random.default_rng(12), 2000, 8, spread).astype(np.float32)
    q_ref = R.ref_quality(R.RQ_HEX, R.REF_MEAN_RATIO, pts)
    q64 = R.element_metric_f64(R.RQ_HEX, R.REF_MEAN_RATIO, pts)
    _assert_close(q_ref, q64, MR_TOL)
    if spread > 0.5:
        assert (q_ref == 0).mean() > 0.05        # the det < eps branch is exercised


def test_oracle_triangle_and_quad_metrics_match_reference(ref):
    R = ref
    rng = np.random.default_rng(13)
    tri = _random_elements(rng, 3000, 3, 0.35).astype(np.float32)
    tri2 = tri.copy()
    tri2[:, :, 2] = 0
    good = np.abs(R.element_metric_f64(R.RQ_TRI2D, R.REF_MEAN_RATIO, tri2)) > 0.05
    for crit in _crits(R):
        for fn, p in ((R.RQ_TRI2D, tri2), (R.RQ_TRI, tri)):
            q_ref = R.ref_quality(fn, crit, p)
            q64 = R.element_metric_f64(fn, crit, p)
            sel = slice(None) if crit == R.REF_MEAN_RATIO else good
            _assert_close(q_ref[sel], q64[sel], _tol(R, crit))
    # normal-signed surface metrics: the normal of the unperturbed element, tilted at random
    n = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0]).astype(np.float64)
    n = n / np.linalg.norm(n, axis=1, keepdims=True) + rng.normal(0, 0.8, size=n.shape)
    n = (n / np.linalg.norm(n, axis=1, keepdims=True)).astype(np.float32)
    for crit in _crits(R):
        q_ref = R.ref_quality(R.RQ_TRI_N, crit, tri, n)
        q64 = R.element_metric_f64(R.RQ_TRI_N, crit, tri, n)
        sel = slice(None) if crit == R.REF_MEAN_RATIO else good
        _assert_close(q_ref[sel], q64[sel], _tol(R, crit))
    quad = _random_elements(rng, 3000, 8, 0.15)[:, :4].astype(np.float32)
    qn = np.cross(quad[:, 1] - quad[:, 0], quad[:, 3] - quad[:, 0]).astype(np.float64)
    qn = qn / np.linalg.norm(qn, axis=1, keepdims=True) + rng.normal(0, 0.5, size=qn.shape)
    qn = (qn / np.linalg.norm(qn, axis=1, keepdims=True)).astype(np.float32)
    _assert_close(R.ref_quality(R.RQ_QUAD, R.REF_MEAN_RATIO, quad),
                  R.element_metric_f64(R.RQ_QUAD, R.REF_MEAN_RATIO, quad), MR_TOL)
    q_ref = R.ref_quality(R.RQ_QUAD_N, R.REF_MEAN_RATIO, quad, qn)
    q64 = R.element_metric_f64(R.RQ_QUAD_N, R.REF_MEAN_RATIO, quad, qn)
    # the 0.7 threshold on the sub-triangle normals decides -1: away from it the values agree
    e = quad[:, [1, 2, 3, 0]].astype(np.float64) - quad
    t1, t2 = np.cross(e[:, 1], -e[:, 0]), np.cross(e[:, 3], -e[:, 2])
    d = np.stack([np.einsum("ij,ij->i", t / np.linalg.norm(t, axis=1, keepdims=True), qn) for t in (t1, t2)])
    clear = np.all(np.abs(d - 0.7) > 1e-4, axis=0)
    assert clear.mean() > 0.99
    _assert_close(q_ref[clear], q64[clear], MR_TOL)
    assert (q_ref == -1).mean() > 0.05


def _check_library(vsdmo, R, gm, opt, fn, crit):
    el = gm.array(vsdmo.A_ELEMS).reshape(gm.info["nE"], -1)
    x = gm.positions()
    q_lib = opt.getElementQualities()
    q_ref = R.ref_quality(fn, crit, x[el])
    _assert_close(q_lib, q_ref.astype(np.float64), _tol(R, crit))
    return q_lib


@pytest.mark.parametrize("crit_i", [0, 1, 2])
def test_library_tet_qualities_match_reference(ref, vsdmo, crit_i):
    R = ref
    crit = _crits(R)[crit_i]
    xyz, tets = G.tet_cube(8, seed=3, jitter=0.45)
    gm = vsdmo.DMOMeshTet(xyz, tets)
    opt = vsdmo.DMOTetClass(gm, _lib_crit(vsdmo, R, crit), 0.5, 2)
    _check_library(vsdmo, R, gm, opt, R.RQ_TET, crit)
    opt.optimize()
    _check_library(vsdmo, R, gm, opt, R.RQ_TET, crit)


def test_library_hex_qualities_match_reference(ref, vsdmo):
    R = ref
    xyz, hexes = G.hex_cube(6, seed=3, jitter=0.35)
    gm = vsdmo.DMOMeshHex(xyz, hexes)
    opt = vsdmo.DMOHexClass(gm, vsdmo.QualityCriterium.MEAN_RATIO, 0.5, 2)
    _check_library(vsdmo, R, gm, opt, R.RQ_HEX, R.REF_MEAN_RATIO)
    opt.optimize()
    _check_library(vsdmo, R, gm, opt, R.RQ_HEX, R.REF_MEAN_RATIO)


@pytest.mark.parametrize("crit_i", [0, 1, 2])
def test_library_triangle_qualities_match_reference(ref, vsdmo, crit_i):
    R = ref
    crit = _crits(R)[crit_i]
    xyz, tri = G.tri_grid(16, seed=5)
    gm = vsdmo.DMOMeshTri(xyz, tri)
    opt = vsdmo.DMOTriFlatClass(gm, _lib_crit(vsdmo, R, crit), 0.5, 2)
    _check_library(vsdmo, R, gm, opt, R.RQ_TRI2D, crit)
    opt.optimize()
    _check_library(vsdmo, R, gm, opt, R.RQ_TRI2D, crit)
    xyz, tri = G.config3_tri(seed=2, level=3)
    gm = vsdmo.DMOMeshTri(xyz, tri)
    opt = vsdmo.DMOTriClass(gm, _lib_crit(vsdmo, R, crit), 0.5, 2)
    _check_library(vsdmo, R, gm, opt, R.RQ_TRI, crit)


def test_library_quad_qualities_match_reference(ref, vsdmo):
    R = ref
    xyz, quads = G.config3_quad(seed=2, nu=32, nv=16)
    gm = vsdmo.DMOMeshQuad(xyz, quads)
    opt = vsdmo.DMOQuadClass(gm, vsdmo.QualityCriterium.MEAN_RATIO, 0.5, 2)
    _check_library(vsdmo, R, gm, opt, R.RQ_QUAD, R.REF_MEAN_RATIO)
    opt.optimize()
    _check_library(vsdmo, R, gm, opt, R.RQ_QUAD, R.REF_MEAN_RATIO)
