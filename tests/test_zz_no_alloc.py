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
