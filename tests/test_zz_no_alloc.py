"""The allocation-free quality reduction (vsdmo_quality_reduce_noalloc).

Some callers cannot allocate device memory: an engine that hands this library a fixed arena,
or code that runs where cudaMalloc / cudaFree are forbidden or would stall the device. For
them the library keeps the reduction's per-block scratch in a fixed device array. This test
calls that entry point through the C ABI twice in a row (the second call reuses the scratch
the first one left behind) and checks both results against the optimiser's existing
quality entry points. It lives in its own file, collected last, and passes both alone in a
fresh process and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from volumesurfacediscretemeshoptimization_b200 import meshgen as G

pytestmark = pytest.mark.gpu

TOL = 2e-6  # same tolerance as the quality comparisons in test_gpu_parity.py


def _run_noalloc(lib, elem_type, flat, d_xyz, nV, d_el, nE, thr, out_min, out_sum, out_below, stream):
    return lib.vsdmo_quality_reduce_noalloc(elem_type, flat, C.c_void_p(d_xyz.data_ptr()), nV,
                                            C.c_void_p(d_el.data_ptr()), nE, thr,
                                            C.c_void_p(out_min.data_ptr()), C.c_void_p(out_sum.data_ptr()),
                                            C.c_void_p(out_below.data_ptr()), C.c_void_p(stream))


@pytest.mark.parametrize("case", ["tet", "tri_flat"])
def test_no_alloc_reduction_matches_existing_entry_points(vsdmo, case):
    import torch
    from volumesurfacediscretemeshoptimization_b200 import _capi
    lib = _capi.lib()
    if case == "tet":
        xyz, el = G.tet_cube(14, seed=6)
        mesh = vsdmo.DMOMeshTet(xyz, el)
        opt = vsdmo.DMOTetClass(mesh, n_iter=2)
        et, flat = _capi.TET, 0
    else:
        xyz, el = G.tri_grid(40, seed=8)
        mesh = vsdmo.DMOMeshTri(xyz, el)
        opt = vsdmo.DMOTriFlatClass(mesh, n_iter=2)
        et, flat = _capi.TRI, 1
    opt.optimize()                       # reduce something other than the initial state
    ref_min, ref_mean = opt.quality_stats()
    q = opt.getElementQualities()
    thr = float(np.median(q))
    ref_below = int((q < thr).sum())
    x_now = mesh.positions(original_order=True)
    dev = torch.device("cuda", 0)
    d_xyz = torch.from_numpy(x_now).to(dev).contiguous()
    d_el = torch.from_numpy(el).to(dev).contiguous()
    out_min = torch.empty(1, dtype=torch.float32, device=dev)
    out_sum = torch.empty(1, dtype=torch.float64, device=dev)
    out_below = torch.empty(1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        out_min.fill_(float("nan"))
        out_sum.fill_(float("nan"))
        out_below.fill_(-1)
        st = _run_noalloc(lib, et, flat, d_xyz, len(xyz), d_el, len(el), thr, out_min, out_sum, out_below, stream)
        assert st == 0, lib.vsdmo_last_error()
        torch.cuda.synchronize(dev)
        got_min = float(out_min.item())
        got_mean = float(out_sum.item()) / len(el)
        assert abs(got_min - ref_min) <= TOL, (call, got_min, ref_min)
        assert abs(got_mean - ref_mean) <= TOL, (call, got_mean, ref_mean)
        assert int(out_below.item()) == ref_below, (call, int(out_below.item()), ref_below)


def test_no_alloc_rejects_oversized_meshes(vsdmo):
    import torch
    from volumesurfacediscretemeshoptimization_b200 import _capi
    lib = _capi.lib()
    dev = torch.device("cuda", 0)
    d = torch.zeros(16, dtype=torch.float32, device=dev)
    di = torch.zeros(16, dtype=torch.int32, device=dev)
    dd = torch.zeros(1, dtype=torch.float64, device=dev)
    st = _run_noalloc(lib, _capi.TET, 0, d, 4, di, 8_388_609, 0.5, d, dd, di, 0)
    assert st == _capi.E_ARG
    assert b"8388608" in lib.vsdmo_last_error()


def _outputs(dev):
    import torch
    return (torch.empty(1, dtype=torch.float32, device=dev), torch.empty(1, dtype=torch.float64, device=dev),
            torch.empty(1, dtype=torch.int32, device=dev))


def test_no_alloc_skips_elements_outside_the_mesh(vsdmo):
    """One index past the last vertex and one negative index: nothing outside the caller's
    arrays is read, the results say so (-1 and NaN), and the next call is correct again."""
    import torch
    from volumesurfacediscretemeshoptimization_b200 import _capi
    lib = _capi.lib()
    xyz, el = G.tet_cube(6, seed=3)
    mesh = vsdmo.DMOMeshTet(xyz, el)
    ref_min, ref_mean = vsdmo.DMOTetClass(mesh, n_iter=1).quality_stats()
    dev = torch.device("cuda", 0)
    d_xyz = torch.from_numpy(xyz).to(dev).contiguous()
    bad = el.copy()
    bad[5, 2] = len(xyz)
    bad[9, 0] = -3
    d_bad = torch.from_numpy(bad).to(dev).contiguous()
    d_el = torch.from_numpy(el).to(dev).contiguous()
    out_min, out_sum, out_below = _outputs(dev)
    st = _run_noalloc(lib, _capi.TET, 0, d_xyz, len(xyz), d_bad, len(el), 0.5, out_min, out_sum, out_below, 0)
    assert st == 0, lib.vsdmo_last_error()
    torch.cuda.synchronize(dev)
    assert int(out_below.item()) == -1
    assert np.isnan(float(out_min.item())) and np.isnan(float(out_sum.item()))
    st = _run_noalloc(lib, _capi.TET, 0, d_xyz, len(xyz), d_el, len(el), 0.5, out_min, out_sum, out_below, 0)
    assert st == 0, lib.vsdmo_last_error()
    torch.cuda.synchronize(dev)
    assert abs(float(out_min.item()) - ref_min) <= TOL
    assert abs(float(out_sum.item()) / len(el) - ref_mean) <= TOL
    assert int(out_below.item()) >= 0


def test_no_alloc_large_mesh_with_clamped_blocks(vsdmo):
    """4.37 M tetrahedra: more than 256 threads x 32 elements x 1024 blocks / 2, so the grid is
    clamped to its 1024 blocks and every thread strides over more than 16 elements."""
    import torch
    from volumesurfacediscretemeshoptimization_b200 import _capi
    lib = _capi.lib()
    xyz, el = G.tet_cube(90, seed=4)
    assert len(el) > 256 * 32 * 1024 // 2
    mesh = vsdmo.DMOMeshTet(xyz, el)
    ref_min, ref_mean = vsdmo.DMOTetClass(mesh, n_iter=1).quality_stats()
    dev = torch.device("cuda", 0)
    d_xyz = torch.from_numpy(xyz).to(dev).contiguous()
    d_el = torch.from_numpy(el).to(dev).contiguous()
    out_min, out_sum, out_below = _outputs(dev)
    for _ in range(2):
        st = _run_noalloc(lib, _capi.TET, 0, d_xyz, len(xyz), d_el, len(el), 0.5, out_min, out_sum, out_below, 0)
        assert st == 0, lib.vsdmo_last_error()
        torch.cuda.synchronize(dev)
        assert abs(float(out_min.item()) - ref_min) <= TOL
        assert abs(float(out_sum.item()) / len(el) - ref_mean) <= TOL


def test_no_alloc_accepts_the_limit(vsdmo):
    """Exactly 8,388,608 elements (all corners at vertex 0) is accepted and runs."""
    import torch
    from volumesurfacediscretemeshoptimization_b200 import _capi
    lib = _capi.lib()
    dev = torch.device("cuda", 0)
    n = 8_388_608
    d_xyz = torch.zeros(12, dtype=torch.float32, device=dev)
    d_el = torch.zeros(4 * n, dtype=torch.int32, device=dev)
    out_min, out_sum, out_below = _outputs(dev)
    st = _run_noalloc(lib, _capi.TET, 0, d_xyz, 4, d_el, n, 0.5, out_min, out_sum, out_below, 0)
    assert st == 0, lib.vsdmo_last_error()
    torch.cuda.synchronize(dev)
    assert int(out_below.item()) == 0   # degenerate tetrahedra give NaN qualities, never below
