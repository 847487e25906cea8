"""Meshes with one very high-valence vertex (fans and stars of thousands of elements).

The build orders each vertex's short rows (its halfedges, its adjacency pairs, the faces it
starts) with one warp per row, in time quadratic in the row's length. A row longer than 4096
entries switches the generic row sorts to radix sorts (same arrays); the halfedge fan walk and the
tetrahedron face pairing refuse such a mesh with VSDMO_E_VALENCE instead. Either way the build
ends in bounded time, never in a warp scanning a row of a million entries.
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TRI, TET = 0, 2


def tri_fan(n):
    """A flat disk: vertex 0 at the centre joined to n rim vertices (n triangles)."""
    a = 2 * np.pi * np.arange(n) / n
    xyz = np.zeros((n + 1, 3), np.float32)
    xyz[1:, 0] = np.cos(a)
    xyz[1:, 1] = np.sin(a)
    k = np.arange(n)
    tris = np.stack([np.zeros(n, np.int64), 1 + k, 1 + (k + 1) % n], 1).astype(np.int32)
    return xyz, tris


def tri_disk2(n):
    """A flat disk of two rings: vertex 0 at the centre joined to n inner-ring vertices, an
    annulus of 2n triangles to n outer-ring (boundary) vertices. The centre and the inner ring
    are free vertices, so the centre's row of colouring pairs holds 2n entries."""
    a = 2 * np.pi * np.arange(n) / n
    xyz = np.zeros((2 * n + 1, 3), np.float32)
    xyz[1:n + 1, 0], xyz[1:n + 1, 1] = 0.5 * np.cos(a), 0.5 * np.sin(a)
    xyz[n + 1:, 0], xyz[n + 1:, 1] = np.cos(a), np.sin(a)
    k = np.arange(n)
    i0, i1 = 1 + k, 1 + (k + 1) % n
    o0, o1 = n + 1 + k, n + 1 + (k + 1) % n
    tris = np.concatenate([np.stack([np.zeros(n, np.int64), i0, i1], 1),
                           np.stack([i0, o0, o1], 1), np.stack([i0, o1, i1], 1)]).astype(np.int32)
    return xyz, tris


def tet_star(n_lon, n_lat):
    """Vertex 0 inside a closed UV sphere, joined to each of its 2 n_lon (n_lat - 1) triangles."""
    v = [[0.05, 0.03, 0.02], [0.0, 0.0, 1.0]]
    for i in range(1, n_lat):
        th = np.pi * i / n_lat
        for j in range(n_lon):
            ph = 2 * np.pi * j / n_lon
            v.append([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])
    v.append([0.0, 0.0, -1.0])
    ring = lambda i, j: 2 + (i - 1) * n_lon + (j % n_lon)
    t = [[1, ring(1, j), ring(1, j + 1)] for j in range(n_lon)]
    for i in range(1, n_lat - 1):
        for j in range(n_lon):
            a, b, c, d = ring(i, j), ring(i + 1, j), ring(i + 1, j + 1), ring(i, j + 1)
            t += [[a, b, c], [a, c, d]]
    s = len(v) - 1
    t += [[s, ring(n_lat - 1, j + 1), ring(n_lat - 1, j)] for j in range(n_lon)]
    tets = np.array([[0, a, c, b] for a, b, c in t], np.int32)
    return np.array(v, np.float32), tets


@pytest.mark.parametrize("gen", ["fan3000", "disk2500"])
def test_high_valence_disks_build_bit_exact(oracle_mod, vsdmo, gen):
    """fan3000: the centre's halfedge row holds 3000 entries (one warp per row); disk2500: its row
    of colouring pairs holds 5000 (over 4096: the radix-sorted path)."""
    xyz, tris = tri_fan(3000) if gen == "fan3000" else tri_disk2(2500)
    t0 = time.perf_counter()
    gm = vsdmo.DMOMeshTri(xyz, tris)
    dt = time.perf_counter() - t0
    assert dt < 10.0, dt
    assert gm.info["maxNumHalfedges"] == (3000 if gen == "fan3000" else 2500)   # the centre's fan
    om = oracle_mod.OracleMesh(TRI, xyz, tris)
    assert om.info == gm.info
    A, B = om.arrays(), gm.arrays()
    for k in A:
        if A[k].dtype == np.float32:
            na = np.isnan(A[k])
            assert np.array_equal(na, np.isnan(B[k])), k
            assert np.array_equal(A[k][~na].view(np.uint32), B[k][~na].view(np.uint32)), k
        else:
            assert np.array_equal(A[k], B[k]), k
    # the centre's ring is far over the flat kernel's budget: the optimiser refuses it
    with pytest.raises(vsdmo.VSDMOError) as e:
        vsdmo.DMOTriFlatClass(gm)
    assert e.value.status == 4  # VSDMO_E_VALENCE


def test_fan_of_5000_triangles_is_refused_quickly(vsdmo):
    xyz, tris = tri_fan(5000)
    t0 = time.perf_counter()
    with pytest.raises(vsdmo.VSDMOError) as e:
        vsdmo.DMOMeshTri(xyz, tris)
    assert e.value.status == 4  # VSDMO_E_VALENCE
    assert time.perf_counter() - t0 < 10.0
    # the library stays usable
    xyz, tris = tri_fan(12)
    assert vsdmo.DMOMeshTri(xyz, tris).info["nE"] == 12


def test_star_of_2400_tetrahedra_is_refused_quickly(vsdmo):
    xyz, tets = tet_star(40, 31)           # 2 * 40 * 30 = 2400 tetrahedra around vertex 0
    assert len(tets) == 2400
    t0 = time.perf_counter()
    with pytest.raises(vsdmo.VSDMOError) as e:
        vsdmo.DMOMeshTet(xyz, tets)
    assert e.value.status == 4  # VSDMO_E_VALENCE
    assert time.perf_counter() - t0 < 10.0


def test_star_of_1200_tetrahedra_builds_bit_exact(oracle_mod, vsdmo):
    xyz, tets = tet_star(30, 21)           # 1200 tetrahedra around vertex 0: 3600 faces it starts
    assert len(tets) == 1200
    gm = vsdmo.DMOMeshTet(xyz, tets)
    om = oracle_mod.OracleMesh(TET, xyz, tets)
    assert om.info == gm.info
    A, B = om.arrays(), gm.arrays()
    for k in A:
        if A[k].dtype == np.float32:
            na = np.isnan(A[k])
            assert np.array_equal(A[k][~na].view(np.uint32), B[k][~na].view(np.uint32)), k
        else:
            assert np.array_equal(A[k], B[k]), k
