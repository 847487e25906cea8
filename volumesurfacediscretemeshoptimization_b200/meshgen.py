"""Seeded synthetic meshes that stand in for the reference's input files.

The reference ships no sample meshes (its ``res/`` directory holds shaders only), so
every workload here is generated: structured grids, Kuhn-subdivided cubes, hex cubes,
an icosphere and a quad torus, each with a seeded perturbation of the free vertices.
All generators return ``(xyz, elems)`` as ``float32 [nV, 3]`` and ``int32 [nE, k]``
numpy arrays in the element orientation the reference expects:

* triangles counter-clockwise (positive 2D area, outward normal on closed surfaces),
  as read by ``io/ParserOFF.cu:16-88``;
* tetrahedra with ``(v1-v0) . ((v2-v0) x (v3-v0)) > 0`` (TetGen node order, the order
  ``dmo/DMOQualityTet.h:119-143`` treats as positive volume);
* hexahedra in the OpenVolumeMesh corner order of ``mesh/MeshGPUCommon.cu:1334-1369``
  (bottom face 0-1-2-3 counter-clockwise seen from below... i.e. 0,1,2,3 then 4,5,6,7 above
  them with 4 over 0, 5 over 3, 6 over 2, 7 over 1, which keeps ``shapeMetricHex`` positive);
* quads counter-clockwise.

Random numbers come from ``numpy.random.default_rng(seed)`` (PCG64).
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "tri_grid", "tet_cube", "hex_cube", "icosphere", "torus_quads",
    "perturb_interior", "config1", "config2", "config2_hex", "config3_tri",
    "config3_quad", "config5",
]


def _rng(seed):
    return np.random.default_rng(seed)


def tri_grid(n: int = 64, seed: int | None = 0, jitter: float = 0.4):
    """``n x n`` vertex grid on the unit square, each cell split along its (0,0)-(1,1)
    diagonal into two counter-clockwise triangles; interior vertices displaced by
    ``U(-jitter*h, jitter*h)`` per axis (``h = 1/(n-1)``), boundary vertices exact, z = 0.
    Vertex ``(i, j)`` (x index ``i``, y index ``j``) has index ``j*n + i``."""
    h = 1.0 / (n - 1)
    j, i = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    xyz = np.zeros((n * n, 3), dtype=np.float64)
    xyz[:, 0] = (i * h).ravel()
    xyz[:, 1] = (j * h).ravel()
    cj, ci = np.meshgrid(np.arange(n - 1), np.arange(n - 1), indexing="ij")
    v00 = (cj * n + ci).ravel()
    v10 = v00 + 1
    v01 = v00 + n
    v11 = v00 + n + 1
    t1 = np.stack([v00, v10, v11], 1)
    t2 = np.stack([v00, v11, v01], 1)
    tris = np.empty((2 * len(v00), 3), dtype=np.int64)
    tris[0::2] = t1
    tris[1::2] = t2
    if seed is not None and jitter > 0:
        inner = ((i > 0) & (i < n - 1) & (j > 0) & (j < n - 1)).ravel()
        r = _rng(seed).uniform(-jitter * h, jitter * h, size=(inner.sum(), 2))
        xyz[inner, :2] += r
    return xyz.astype(np.float32), tris.astype(np.int32)


def quad_grid(n: int = 64, seed: int | None = 0, jitter: float = 0.4):
    """``n x n`` vertex grid on the unit square as counter-clockwise quads, interior vertices
    displaced by ``U(-jitter*h, jitter*h)`` per axis, boundary exact, z = 0."""
    h = 1.0 / (n - 1)
    j, i = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    xyz = np.zeros((n * n, 3), dtype=np.float64)
    xyz[:, 0] = (i * h).ravel()
    xyz[:, 1] = (j * h).ravel()
    cj, ci = np.meshgrid(np.arange(n - 1), np.arange(n - 1), indexing="ij")
    v00 = (cj * n + ci).ravel()
    quads = np.stack([v00, v00 + 1, v00 + n + 1, v00 + n], 1)
    if seed is not None and jitter > 0:
        inner = ((i > 0) & (i < n - 1) & (j > 0) & (j < n - 1)).ravel()
        r = _rng(seed).uniform(-jitter * h, jitter * h, size=(inner.sum(), 2))
        xyz[inner, :2] += r
    return xyz.astype(np.float32), quads.astype(np.int32)


_KUHN = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]


def tet_cube(n: int = 48, seed: int | None = 0, jitter: float = 0.3):
    """Unit cube with ``n^3`` cells, each split into the 6 Kuhn tetrahedra along its
    main diagonal. Interior vertices displaced by ``U(-jitter*h, jitter*h)`` per axis.
    Vertex ``(i, j, k)`` has index ``(k*(n+1) + j)*(n+1) + i``."""
    m = n + 1
    h = 1.0 / n
    k, j, i = np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij")
    xyz = np.stack([i.ravel() * h, j.ravel() * h, k.ravel() * h], 1).astype(np.float64)
    ck, cj, ci = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    base = ((ck * m + cj) * m + ci).ravel()
    step = np.array([1, m, m * m], dtype=np.int64)
    tets = np.empty((len(base), 6, 4), dtype=np.int64)
    for t, perm in enumerate(_KUHN):
        a = base
        b = a + step[perm[0]]
        c = b + step[perm[1]]
        d = c + step[perm[2]]
        tets[:, t] = np.stack([a, b, c, d], 1)
    tets = tets.reshape(-1, 4)
    # orient positively: (v1-v0).((v2-v0)x(v3-v0)) > 0 on the unperturbed lattice
    p = xyz[tets]
    det = np.einsum("ij,ij->i", p[:, 1] - p[:, 0], np.cross(p[:, 2] - p[:, 0], p[:, 3] - p[:, 0]))
    neg = det < 0
    tets[neg, 1], tets[neg, 2] = tets[neg, 2].copy(), tets[neg, 1].copy()
    if seed is not None and jitter > 0:
        inner = ((i > 0) & (i < n) & (j > 0) & (j < n) & (k > 0) & (k < n)).ravel()
        r = _rng(seed).uniform(-jitter * h, jitter * h, size=(inner.sum(), 3))
        xyz[inner] += r
    return xyz.astype(np.float32), tets.astype(np.int32)


def hex_cube(n: int = 32, seed: int | None = 0, jitter: float = 0.3):
    """Unit cube with ``n^3`` hexahedra. Corner order per cell (offsets in cells):
    0=(0,0,1) 1=(1,0,1) 2=(1,1,1) 3=(0,1,1) 4=(0,0,0) 5=(1,0,0) 6=(1,1,0) 7=(0,1,0): the
    order under which every sub-tetrahedron of the reference's shapeMetricHex
    (dmo/DMOQualityHex.h:54-71, which reads the corners as 4 5 6 7 0 1 2 3) is positive, the
    metric of an undistorted cube is 1 and the six faces of k_constructQuadsFromHexahedra
    (mesh/MeshGPUCommon.cu:1412-1430) point outwards."""
    m = n + 1
    h = 1.0 / n
    k, j, i = np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij")
    xyz = np.stack([i.ravel() * h, j.ravel() * h, k.ravel() * h], 1).astype(np.float64)
    ck, cj, ci = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    b = ((ck * m + cj) * m + ci).ravel()
    X, Y, Z = 1, m, m * m
    hexes = np.stack([b + Z, b + X + Z, b + X + Y + Z, b + Y + Z, b, b + X, b + X + Y, b + Y], 1)
    if seed is not None and jitter > 0:
        inner = ((i > 0) & (i < n) & (j > 0) & (j < n) & (k > 0) & (k < n)).ravel()
        r = _rng(seed).uniform(-jitter * h, jitter * h, size=(inner.sum(), 3))
        xyz[inner] += r
    return xyz.astype(np.float32), hexes.astype(np.int32)


def icosphere(level: int = 7):
    """Unit icosphere: icosahedron subdivided ``level`` times (edge midpoints pushed to the
    sphere). ``10*4^level + 2`` vertices, ``20*4^level`` outward-oriented triangles."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
                  [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]],
                 dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9],
                  [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2],
                  [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10],
                  [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    for _ in range(level):
        nv = len(v)
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]], 0)
        es = np.sort(e, 1)
        key = es[:, 0] * nv + es[:, 1]
        uk, inv = np.unique(key, return_inverse=True)
        a, b = uk // nv, uk % nv
        mid = v[a] + v[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        m = nv + inv.reshape(3, -1).T  # midpoints of edges 01, 12, 20
        v = np.concatenate([v, mid], 0)
        f0, f1, f2 = f[:, 0], f[:, 1], f[:, 2]
        m01, m12, m20 = m[:, 0], m[:, 1], m[:, 2]
        f = np.concatenate([np.stack([f0, m01, m20], 1), np.stack([f1, m12, m01], 1),
                            np.stack([f2, m20, m12], 1), np.stack([m01, m12, m20], 1)], 0)
    # make every triangle outward
    p = v[f]
    nrm = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
    flip = np.einsum("ij,ij->i", nrm, p.sum(1)) < 0
    f[flip, 1], f[flip, 2] = f[flip, 2].copy(), f[flip, 1].copy()
    return v.astype(np.float32), f.astype(np.int32)


def torus_quads(nu: int = 512, nv: int = 256, R: float = 1.0, r: float = 0.35):
    """Torus with ``nu`` segments around the main circle and ``nv`` around the tube;
    ``nu*nv`` vertices and outward counter-clockwise quads."""
    u = 2 * np.pi * np.arange(nu) / nu
    w = 2 * np.pi * np.arange(nv) / nv
    U, W = np.meshgrid(u, w, indexing="ij")
    x = (R + r * np.cos(W)) * np.cos(U)
    y = (R + r * np.cos(W)) * np.sin(U)
    z = r * np.sin(W)
    xyz = np.stack([x.ravel(), y.ravel(), z.ravel()], 1)
    a, b = np.meshgrid(np.arange(nu), np.arange(nv), indexing="ij")
    idx = lambda ia, ib: (ia % nu) * nv + (ib % nv)
    q = np.stack([idx(a, b), idx(a + 1, b), idx(a + 1, b + 1), idx(a, b + 1)], -1).reshape(-1, 4)
    p = xyz[q]
    nrm = np.cross(p[:, 1] - p[:, 0], p[:, 3] - p[:, 0])
    cen = p.mean(1)
    ring = np.stack([R * np.cos(np.arctan2(cen[:, 1], cen[:, 0])),
                     R * np.sin(np.arctan2(cen[:, 1], cen[:, 0])), np.zeros(len(cen))], 1)
    if np.einsum("ij,ij->i", nrm, cen - ring).mean() < 0:
        q = q[:, ::-1].copy()
    return xyz.astype(np.float32), q.astype(np.int32)


def perturb_surface(xyz, elems, seed: int = 0, tangential: float = 0.35, normal_sigma: float = 1e-3,
                    normal_absolute: bool = False):
    """Tangential noise ``U(-t*l, t*l)`` (``l`` = mean incident edge length) in the tangent
    plane of the area-weighted vertex normal, plus normal noise along it: ``N(0, normal_sigma)``
    with ``normal_absolute``, else ``N(0, normal_sigma * l)``. An absolute sigma of 1e-3 on edges
    of ~0.01 tilts neighbouring faces by more than 20 degrees and turns many vertices into
    feature vertices under the reference's dihedral rule (mesh/MeshTriGPU.cu:506)."""
    xyz = xyz.astype(np.float64)
    k = elems.shape[1]
    nV = len(xyz)
    e = np.concatenate([elems[:, [a, (a + 1) % k]] for a in range(k)], 0)
    length = np.linalg.norm(xyz[e[:, 0]] - xyz[e[:, 1]], axis=1)
    lsum = np.bincount(e[:, 0], length, nV) + np.bincount(e[:, 1], length, nV)
    cnt = np.bincount(e[:, 0], None, nV) + np.bincount(e[:, 1], None, nV)
    lmean = lsum / np.maximum(cnt, 1)
    p = xyz[elems]
    fn = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
    vn = np.zeros_like(xyz)
    for a in range(k):
        np.add.at(vn, elems[:, a], fn)
    vn /= np.linalg.norm(vn, axis=1, keepdims=True)
    ref = np.where(np.abs(vn[:, :1]) < 0.9, np.array([[1.0, 0, 0]]), np.array([[0, 1.0, 0]]))
    t1 = np.cross(vn, ref)
    t1 /= np.linalg.norm(t1, axis=1, keepdims=True)
    t2 = np.cross(vn, t1)
    g = _rng(seed)
    a = g.uniform(-tangential, tangential, size=(nV, 2)) * lmean[:, None]
    nn = g.normal(0.0, normal_sigma, size=nV)
    out = xyz + a[:, :1] * t1 + a[:, 1:] * t2 + (nn if normal_absolute else nn * lmean)[:, None] * vn
    return out.astype(np.float32)


def perturb_interior(xyz, mask, h, jitter, seed):
    xyz = xyz.astype(np.float64).copy()
    r = _rng(seed).uniform(-jitter * h, jitter * h, size=(int(mask.sum()), xyz.shape[1]))
    xyz[mask] += r
    return xyz.astype(np.float32)


# ---- the benchmark workloads -------------------------------------------------------

def config1(seed: int = 0):
    """64x64 flat triangle grid, 4096 vertices / 7938 triangles, jitter 0.4h."""
    return tri_grid(64, seed, 0.4)


def config2(seed: int = 0, n: int = 48):
    """Kuhn tet cube 48^3: 117,649 vertices / 663,552 tetrahedra, jitter 0.3h."""
    return tet_cube(n, seed, 0.3)


def config2_hex(seed: int = 0, n: int = 32):
    """Hex cube 32^3: 35,937 vertices / 32,768 hexahedra, jitter 0.3h."""
    return hex_cube(n, seed, 0.3)


def config3_tri(seed: int = 0, level: int = 7, variant: str = "as_written"):
    """Icosphere level 7 (163,842 vertices / 327,680 triangles), radius 1, with surface noise.

    ``as_written``: tangential noise U(+-0.35 l) and normal noise N(0, 1e-3), absolute, as the
    workload is specified; the normal noise makes many vertices feature vertices under the
    reference's 20 degree dihedral rule, which the feature passes then move along their curves.
    ``feature_free``: tangential 0.3 l and N(0, 1e-3 l), which keeps the sphere free of
    feature vertices (a smooth-surface variant)."""
    v, f = icosphere(level)
    if variant == "as_written":
        return perturb_surface(v, f, seed, tangential=0.35, normal_sigma=1e-3, normal_absolute=True), f
    return perturb_surface(v, f, seed, tangential=0.3), f


def config3_quad(seed: int = 0, nu: int = 512, nv: int = 256, variant: str = "as_written"):
    """Torus R=1, r=0.35 with 512x256 quads and surface noise.

    ``as_written``: tangential U(+-0.35 l) and absolute normal noise N(0, 1e-3), as specified.
    ``feature_free``: tangential 0.2 l and N(0, 1e-3 l): the quads are up to 2:1 anisotropic
    (edges 0.008-0.017) and larger noise folds some of them into feature vertices."""
    v, q = torus_quads(nu, nv)
    if variant == "as_written":
        return perturb_surface(v, q, seed, tangential=0.35, normal_sigma=1e-3, normal_absolute=True), q
    return perturb_surface(v, q, seed, tangential=0.2), q


def config4(seed: int = 0, count: int = 256, v_min: int = 500, v_max: int = 50000):
    """256 independent jittered structured 2D grids, triangles and quads alternating, vertex
    counts log-uniform in [500, 50,000] (grid side round(sqrt(V))), interior jitter 0.4h.
    Returns a list of (elem_type, xyz, elems) with elem_type 0 = triangles, 1 = quads."""
    g = _rng(seed)
    sizes = np.exp(g.uniform(np.log(v_min), np.log(v_max), size=count))
    out = []
    for m, v in enumerate(sizes):
        n = max(4, int(round(np.sqrt(v))))
        if m % 2 == 0:
            xyz, el = tri_grid(n, seed=seed * 1000 + m, jitter=0.4)
            out.append((0, xyz, el))
        else:
            xyz, el = quad_grid(n, seed=seed * 1000 + m, jitter=0.4)
            out.append((1, xyz, el))
    return out


def config5(seed: int = 0, n: int = 100):
    """Kuhn tet cube 100^3: 1,030,301 vertices / 6,000,000 tetrahedra, jitter 0.3h."""
    return tet_cube(n, seed, 0.3)
