"""CPU tests of the C ABI: the shared library loads, exports every entry point include/*.h
declares, and the host-only calls (defaults, status strings, argument validation that
fails before any device work) behave. No kernel runs here."""
import ctypes as C
import glob
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        names.update(re.findall(r"VSDMO_API\s+[\w\s\*]+?\b(vsdmo_\w+)\s*\(", txt))
    return sorted(names)


def test_header_declares_entry_points():
    syms = _declared_symbols()
    assert "vsdmo_mesh_create" in syms and "vsdmo_opt_iterate" in syms
    assert len(syms) >= 25


def test_library_exports_every_declared_symbol(vsdmo):
    from volumesurfacediscretemeshoptimization_b200 import _capi
    lib = _capi.lib()
    missing = [s for s in _declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert set(_capi.EXPORTED) <= set(_declared_symbols())
    out = subprocess.run(["nm", "-D", "--defined-only", _capi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (vsdmo_\w+)", out))
    assert set(_declared_symbols()) <= exported


def test_host_only_calls(vsdmo):
    from volumesurfacediscretemeshoptimization_b200 import _capi
    lib = _capi.lib()
    assert b"sm_100a" in lib.vsdmo_version()
    p = _capi.Params()
    assert lib.vsdmo_params_default(_capi.TET, C.byref(p)) == 0
    assert (p.grid_n, p.depth, p.n_iter, p.fit_ring) == (8, 3, 30, 1)
    assert abs(p.grid_scale - 0.5) < 1e-7
    assert lib.vsdmo_params_default(99, C.byref(p)) == _capi.E_ARG
    assert lib.vsdmo_status_string(_capi.E_MONOTONE) == b"quality decreased"
    h = C.c_void_p()
    # argument errors are reported before any CUDA call
    assert lib.vsdmo_mesh_create(_capi.TET, None, 0, None, 0, 0, 1, None, C.byref(h)) == _capi.E_ARG
    assert b"empty" in lib.vsdmo_last_error()
    assert lib.vsdmo_mesh_create(7, C.c_void_p(1), 1, C.c_void_p(1), 1, 0, 1, None, C.byref(h)) == _capi.E_ARG
    assert b"element type" in lib.vsdmo_last_error()
    assert lib.vsdmo_mesh_create(_capi.HEX, C.c_void_p(1), 1, C.c_void_p(1), 1, 5, 1, None, C.byref(h)) == _capi.E_ARG
    assert lib.vsdmo_opt_iterate(None, 1) == _capi.E_ARG
    # batched meshes: argument errors before any CUDA call
    import numpy as np
    b = C.c_void_p()
    one = np.ones(1, np.int32)
    tet = np.full(1, _capi.TET, np.int32)
    ptr = lambda a: a.ctypes.data_as(C.c_void_p)
    assert lib.vsdmo_batch_create(0, None, None, None, None, None, 0, 1, None, C.byref(b)) == _capi.E_ARG
    assert lib.vsdmo_batch_create(1, ptr(tet), ptr(one), ptr(one), C.c_void_p(1), C.c_void_p(1), 0, 1, None,
                                  C.byref(b)) == _capi.E_ARG
    assert b"VSDMO_TRI or VSDMO_QUAD" in lib.vsdmo_last_error()
    assert lib.vsdmo_batch_info(None, 0) == -1
    assert lib.vsdmo_batch_iterate(None, 1) == _capi.E_ARG


def test_python_api_raises_on_error(vsdmo):
    with pytest.raises(vsdmo.VSDMOError):
        vsdmo._capi.check(vsdmo._capi.E_ARG)
