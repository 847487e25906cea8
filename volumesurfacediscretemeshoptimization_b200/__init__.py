"""B200-native discrete mesh optimisation (DMO) with the reference's mesh / optimizer API.

Python mirror of the reference's C++ interface (DanielZint/VolumeSurfaceDiscreteMeshOptimization):

* ``DMOMeshTriFactory.create(points, tris)`` / ``DMOMeshTetFactory.create(points, tets)``
  -- ``mesh/MeshFactory.h:17-40`` (device-array overloads; file parsing is separate);
* ``DMOTetClass(mesh, QualityCriterium.MEAN_RATIO, gridScale=0.5, n_iter=30)``,
  ``DMOTriFlatClass(...)``, ``DMOTriClass(...)`` and ``DMOQuadClass(...)`` --
  ``dmo/DMOTet.h:21-62``, ``dmo/DMOTriFlat.h:19-51``, ``dmo/DMOTri.h``, ``dmo/DMOQuad.h`` with
  ``optimize()``, ``doIteration()``, ``isDone()``, ``getQuality()``, ``findMinimumQuality()``,
  ``getElementQualities()``, ``getQualityHistogram()``, ``displayQualityGPU()``
  (``dmo/DMOBase.h:23-88``).

Everything runs in ``lib/libvsdmo.so`` through the C ABI of ``include/vsdmo.h``; this module
only marshals arguments. Differences from the reference: meshes are built from arrays you
pass (host numpy or device pointers), vertex numbering is reported through
``permutation()`` / ``positions(original_order=True)``, errors raise ``VSDMOError`` instead of
exiting, and ``fix_boundary`` selects the boundary-fixed runs of the benchmark configs.

``ProposalModel`` and ``DMOTetClass.set_model`` add the learned proposal, which has no
counterpart in the reference.
"""
from __future__ import annotations

import ctypes as C
import os
import enum
import sys


import numpy as np

from . import _capi
from ._capi import VSDMOError, Params, check

__all__ = ["QualityCriterium", "DMOMeshTri", "DMOMeshQuad", "DMOMeshTet", "DMOMeshHex", "DMOMeshTriFactory",
           "DMOMeshQuadFactory", "DMOMeshTetFactory", "DMOMeshHexFactory", "DMOTetClass", "DMOHexClass",
           "DMOTriFlatClass", "DMOTriClass", "DMOQuadClass", "DMOQuadFlatClass", "BatchDMO", "ProposalModel",
           "VSDMOError", "Params", "default_params", "version", "read_mesh_file", "write_mesh_file",
           "COLOR_REFERENCE", "COLOR_ROUNDS"]

A_XYZ, A_NEW_OF_OLD, A_ELEMS, A_SURF_TRIS, A_HE_ROWPTR, A_HALFEDGES, A_HF_ROWPTR, A_HALFFACES, \
    A_COL_FREE, A_COL_FEATURE, A_COL_INNER, A_IS_BOUNDARY1D, A_IS_FEATURE, A_IS_BOUNDARY2D, \
    A_FACE_NORMALS, A_VERTEX_NORMALS = range(16)
ARRAY_NAMES = {A_XYZ: "xyz", A_NEW_OF_OLD: "new_of_old", A_ELEMS: "elems", A_SURF_TRIS: "surf_tris",
               A_HE_ROWPTR: "he_rowptr", A_HALFEDGES: "halfedges", A_HF_ROWPTR: "hf_rowptr",
               A_HALFFACES: "halffaces", A_COL_FREE: "col_free", A_COL_FEATURE: "col_feature",
               A_COL_INNER: "col_inner", A_IS_BOUNDARY1D: "is_boundary1d", A_IS_FEATURE: "is_feature",
               A_IS_BOUNDARY2D: "is_boundary2d", A_FACE_NORMALS: "face_normals",
               A_VERTEX_NORMALS: "vertex_normals"}
_F32 = {A_XYZ, A_FACE_NORMALS, A_VERTEX_NORMALS}
_U8 = {A_IS_BOUNDARY1D, A_IS_FEATURE, A_IS_BOUNDARY2D}
I_ELEM_TYPE = 12
# color_seed value selecting the reference's own JPL priorities n - i (VSDMO_COLOR_REFERENCE)
# instead of the seeded hash; the reference's mesh/VertexColoring.cu:107-125. COLOR_ROUNDS | seed
# (VSDMO_COLOR_ROUNDS) keeps the hashed priorities but colours by JPL round like the reference,
# instead of the default smallest colour free among the higher-priority neighbours.
COLOR_REFERENCE = 0xFFFFFFFF
COLOR_ROUNDS = 0x80000000
INFO_NAMES = ["nV", "nE", "nSurf", "nFeature", "nTris", "nHE", "nColorsFree", "nColorsFeature",
              "nColorsInner", "maxNumHalfedges", "maxNumTetrahedra", "isFlat"]


class QualityCriterium(enum.IntEnum):
    """``DMO::QualityCriterium`` (``dmo/DMOQualityUtil.h:10-18``)."""
    MEAN_RATIO = 0
    AREA = 1
    RIGHT_ANGLE = 2
    JACOBIAN = 3
    MIN_ANGLE = 4
    RADIUS_RATIO = 5
    MAX_ANGLE = 6
    CONDITION = 7   # hex meshes, quad surfaces: inverse condition number of the corner Jacobians (an addition)


def version() -> str:
    return _capi.lib().vsdmo_version().decode()


def default_params(elem_type: int) -> Params:
    p = Params()
    check(_capi.lib().vsdmo_params_default(elem_type, C.byref(p)))
    return p


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class _Mesh:
    elem_type = -1
    k = 0

    def __init__(self, points, elems, color_seed: int = 1, stream=None, device_ptrs=None, handle=None):
        L = _capi.lib()
        h = C.c_void_p()
        if handle is not None:
            h = handle
        elif device_ptrs is not None:
            xyz_ptr, el_ptr, nV, nE = device_ptrs
            check(L.vsdmo_mesh_create(self.elem_type, C.c_void_p(xyz_ptr), nV, C.c_void_p(el_ptr), nE,
                                      _capi.DEVICE, color_seed, C.c_void_p(stream or 0), C.byref(h)))
        else:
            xyz = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)
            el = np.ascontiguousarray(elems, dtype=np.int32).reshape(-1, self.k)
            check(L.vsdmo_mesh_create(self.elem_type, _ptr(xyz), len(xyz), _ptr(el), len(el), _capi.HOST,
                                      color_seed, C.c_void_p(stream or 0), C.byref(h)))
        self.h = h
        self.info = {n: L.vsdmo_mesh_info(h, i) for i, n in enumerate(INFO_NAMES)}
        self.nVertices = self.info["nV"]
        self.nVerticesSurf = self.info["nSurf"]
        self.nVerticesFeature = self.info["nFeature"]

    def close(self):
        if getattr(self, "h", None):
            _capi.lib().vsdmo_mesh_destroy(self.h)
            self.h = None

    def __del__(self, _finalizing=sys.is_finalizing):
        # no library calls while the interpreter shuts down: the CUDA runtime may be gone
        # (bound as a default: module globals are cleared during shutdown)
        if _finalizing():
            return
        try:
            self.close()
        except Exception:
            pass

    def array(self, aid: int) -> np.ndarray:
        L = _capi.lib()
        n = L.vsdmo_mesh_array_len(self.h, aid)
        dt = np.float32 if aid in _F32 else (np.uint8 if aid in _U8 else np.int32)
        out = np.zeros(max(n, 0), dtype=dt)
        if n > 0:
            check(L.vsdmo_mesh_array(self.h, aid, _ptr(out)))
        return out

    def arrays(self) -> dict:
        return {ARRAY_NAMES[a]: self.array(a) for a in ARRAY_NAMES}

    def permutation(self) -> np.ndarray:
        return self.array(A_NEW_OF_OLD)

    def positions(self, original_order: bool = False) -> np.ndarray:
        out = np.zeros((self.nVertices, 3), dtype=np.float32)
        check(_capi.lib().vsdmo_mesh_get_positions(self.h, _ptr(out), int(original_order), _capi.HOST))
        return out

    def set_positions(self, xyz, original_order: bool = False):
        xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
        if len(xyz) != self.nVertices:
            raise ValueError("wrong number of vertices")
        check(_capi.lib().vsdmo_mesh_set_positions(self.h, _ptr(xyz), int(original_order), _capi.HOST))

    def write(self, path: str, fmt: int = _capi.FMT_AUTO):
        """writeOFF / writeTetgen / writeHex (``io/FileWriter.cu``): current positions in the
        caller's numbering."""
        check(_capi.lib().vsdmo_mesh_write_file(self.h, os.fsencode(path), int(fmt)))

    def positions_to_device(self, dev_ptr: int, original_order: bool = True):
        check(_capi.lib().vsdmo_mesh_get_positions(self.h, C.c_void_p(dev_ptr), int(original_order), _capi.DEVICE))


class DMOMeshTri(_Mesh):
    """``DMOMeshTri`` (``mesh/DMOMeshTri.h:81-94``)."""
    elem_type = _capi.TRI
    k = 3


class DMOMeshQuad(_Mesh):
    """``DMOMeshQuad`` (``mesh/DMOMeshQuad.h``): quad surface mesh."""
    elem_type = _capi.QUAD
    k = 4


class DMOMeshTet(_Mesh):
    """``DMOMeshTet`` (``mesh/DMOMeshTet.h:145-198``)."""
    elem_type = _capi.TET
    k = 4


class DMOMeshHex(_Mesh):
    """``DMOMeshHex`` (``mesh/DMOMeshHex.h``): hexahedral volume mesh (corner order of
    ``meshgen.hex_cube``: 0-3 one face, 4-7 the opposite face, 4 below 0)."""
    elem_type = _capi.HEX
    k = 8


_MESH_CLASS = {_capi.TRI: DMOMeshTri, _capi.QUAD: DMOMeshQuad, _capi.TET: DMOMeshTet, _capi.HEX: DMOMeshHex}


def _from_file(path, expect, color_seed, stream):
    """``DMOMesh*Factory::create(filename)`` (``mesh/MeshFactory.cu:3-13,45-55,60-70,101-111``);
    returns None where the reference returns nullptr (the file cannot be opened or parsed)."""
    h = C.c_void_p()
    st = _capi.lib().vsdmo_mesh_create_from_file(os.fsencode(path), _capi.FMT_AUTO, int(color_seed),
                                                  C.c_void_p(stream or 0), C.byref(h))
    if st == _capi.E_IO:
        return None
    check(st)
    got = _capi.lib().vsdmo_mesh_info(h, I_ELEM_TYPE)
    if got != expect:
        _capi.lib().vsdmo_mesh_destroy(h)
        raise VSDMOError(_capi.E_ARG, f"{path} holds element type {got}, this factory builds type {expect}")
    cls = _MESH_CLASS[expect]
    m = cls.__new__(cls)
    _Mesh.__init__(m, None, None, handle=h)
    return m


def read_mesh_file(path, fmt: int = _capi.FMT_AUTO):
    """Host parse of an OFF / TetGen / Medit file: (elem_type, points [n x 3], elems [m x k])."""
    t, nv, ne = C.c_int(), C.c_int(), C.c_int()
    b = os.fsencode(path)
    check(_capi.lib().vsdmo_file_read(b, int(fmt), C.byref(t), C.byref(nv), C.byref(ne), None, None))
    k = {_capi.TRI: 3, _capi.QUAD: 4, _capi.TET: 4, _capi.HEX: 8}[t.value]
    xyz = np.zeros((nv.value, 3), np.float32)
    el = np.zeros((ne.value, k), np.int32)
    check(_capi.lib().vsdmo_file_read(b, int(fmt), C.byref(t), C.byref(nv), C.byref(ne), _ptr(xyz), _ptr(el)))
    return t.value, xyz, el


def write_mesh_file(path, elem_type: int, points, elems, fmt: int = _capi.FMT_AUTO):
    xyz = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    el = np.ascontiguousarray(elems, np.int32)
    check(_capi.lib().vsdmo_file_write(os.fsencode(path), int(fmt), int(elem_type), _ptr(xyz), len(xyz), _ptr(el),
                                       len(el)))


def _surface_of(volume, color_seed, stream, cls):
    h = C.c_void_p()
    check(_capi.lib().vsdmo_mesh_create_surface(volume.h, int(color_seed), C.c_void_p(stream or 0), C.byref(h)))
    m = cls.__new__(cls)
    _Mesh.__init__(m, None, None, handle=h)
    return m


class DMOMeshTriFactory:
    """``DMOMeshTriFactory::create`` (``mesh/MeshFactory.cu:3-41``): from arrays, from an OFF
    file name, or the boundary of a ``DMOMeshTet``."""

    @staticmethod
    def create(points, tris=None, color_seed: int = 1, stream=None):
        if isinstance(points, (str, os.PathLike)):
            return _from_file(points, _capi.TRI, color_seed, stream)
        if isinstance(points, DMOMeshTet):
            return _surface_of(points, color_seed, stream, DMOMeshTri)
        return DMOMeshTri(points, tris, color_seed, stream)


class DMOMeshQuadFactory:
    """``DMOMeshQuadFactory::create`` (``mesh/MeshFactory.cu:60-99``): from arrays, an OFF
    file name, or the boundary of a ``DMOMeshHex``."""

    @staticmethod
    def create(points, quads=None, color_seed: int = 1, stream=None):
        if isinstance(points, (str, os.PathLike)):
            return _from_file(points, _capi.QUAD, color_seed, stream)
        if isinstance(points, DMOMeshHex):
            return _surface_of(points, color_seed, stream, DMOMeshQuad)
        return DMOMeshQuad(points, quads, color_seed, stream)


class DMOMeshHexFactory:
    """``DMOMeshHexFactory::create`` (``mesh/MeshFactory.cu:101-111``): from arrays or a Medit
    file name."""

    @staticmethod
    def create(points, hexes=None, color_seed: int = 1, stream=None):
        if isinstance(points, (str, os.PathLike)):
            return _from_file(points, _capi.HEX, color_seed, stream)
        return DMOMeshHex(points, hexes, color_seed, stream)


class DMOMeshTetFactory:
    """``DMOMeshTetFactory::create`` (``mesh/MeshFactory.cu:45-55``): from arrays or a TetGen
    base name (``base.node`` + ``base.ele``)."""

    @staticmethod
    def create(points, tets=None, color_seed: int = 1, stream=None):
        if isinstance(points, (str, os.PathLike)):
            return _from_file(points, _capi.TET, color_seed, stream)
        return DMOMeshTet(points, tets, color_seed)


class _DMOBase:
    """``DMO::DMOBaseClass`` (``dmo/DMOBase.h:23-88``)."""
    _flat = -1

    def __init__(self, dmo_mesh, qualityCriterium=QualityCriterium.MEAN_RATIO, gridScale: float = 0.5,
                 n_iter: int = 30, fix_boundary: bool = True, use_graph: bool = True, depth: int = 3,
                 check_monotone: bool = True, active_set: bool = False, grid_n: int = 8, fit_ring: int = 1):
        self.mesh = dmo_mesh
        p = default_params(dmo_mesh.elem_type)
        p.quality = int(qualityCriterium)
        p.grid_scale = float(gridScale)
        p.n_iter = int(n_iter)
        p.fix_boundary = int(fix_boundary)
        p.use_graph = int(use_graph)
        p.depth = int(depth)
        p.check_monotone = int(check_monotone)
        p.active_set = int(active_set)
        p.fit_ring = int(fit_ring)
        p.grid_n = int(grid_n)
        p.flat = self._flat
        self.params = p
        h = C.c_void_p()
        check(_capi.lib().vsdmo_opt_create(dmo_mesh.h, C.byref(p), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            _capi.lib().vsdmo_opt_destroy(self.h)
            self.h = None

    def __del__(self, _finalizing=sys.is_finalizing):
        # no library calls while the interpreter shuts down: the CUDA runtime may be gone
        # (bound as a default: module globals are cleared during shutdown)
        if _finalizing():
            return
        try:
            self.close()
        except Exception:
            pass

    def doIteration(self):
        check(_capi.lib().vsdmo_opt_iterate(self.h, 1))

    def iterate(self, n: int):
        check(_capi.lib().vsdmo_opt_iterate(self.h, int(n)))

    def optimize(self):
        check(_capi.lib().vsdmo_opt_optimize(self.h))

    def restart(self):
        """Start over from the mesh's current positions (iteration count 0)."""
        check(_capi.lib().vsdmo_opt_restart(self.h))

    def isDone(self) -> bool:
        return bool(_capi.lib().vsdmo_opt_is_done(self.h))

    @property
    def curr_it(self) -> int:
        return _capi.lib().vsdmo_opt_iterations_done(self.h)

    def getQuality(self) -> float:
        q = C.c_float()
        check(_capi.lib().vsdmo_opt_get_quality(self.h, C.byref(q)))
        return q.value

    def findMinimumQuality(self) -> float:
        q = C.c_float()
        check(_capi.lib().vsdmo_opt_find_min_quality(self.h, C.byref(q), None))
        return q.value

    def quality_stats(self):
        q = C.c_float()
        m = C.c_double()
        check(_capi.lib().vsdmo_opt_find_min_quality(self.h, C.byref(q), C.byref(m)))
        return q.value, m.value

    def getElementQualities(self, out=None):
        """Host numpy array of per-element qualities, or write into a device pointer ``out``."""
        if out is not None:
            check(_capi.lib().vsdmo_opt_element_qualities(self.h, C.c_void_p(out), _capi.DEVICE))
            return None
        q = np.zeros(self.mesh.info["nE"], dtype=np.float32)
        check(_capi.lib().vsdmo_opt_element_qualities(self.h, _ptr(q), _capi.HOST))
        return q

    def getQualityHistogram(self, n_cols: int = 10):
        c = np.zeros(n_cols, dtype=np.int32)
        check(_capi.lib().vsdmo_opt_quality_histogram(self.h, _ptr(c), n_cols))
        return c

    def displayQualityGPU(self, n_cols: int = 10):
        check(_capi.lib().vsdmo_opt_display_quality(self.h, n_cols))

    def history(self):
        n_cap = self.curr_it + 1
        mn = np.zeros(n_cap, dtype=np.float32)
        mean = np.zeros(n_cap, dtype=np.float64)
        n = C.c_int()
        check(_capi.lib().vsdmo_opt_history(self.h, _ptr(mn), _ptr(mean), n_cap, C.byref(n)))
        return mn[: n.value], mean[: n.value]

    def run_color(self, color: int):
        check(_capi.lib().vsdmo_opt_run_color(self.h, int(color)))

    @property
    def launches_per_iteration(self) -> int:
        return _capi.lib().vsdmo_opt_launches_per_iteration(self.h)

    def getLocalSurfacePoints(self, vid: int, nu: int, nv: int, featureSid: int = 0) -> np.ndarray:
        """Samples [nu * nv x 3] of vertex vid's (internal numbering) own local surface."""
        out = np.zeros((nu * nv, 3), np.float32)
        check(_capi.lib().vsdmo_opt_local_surface_points(self.h, int(vid), int(nu), int(nv), _ptr(out), _capi.HOST,
                                                         int(featureSid)))
        return out

    def getEstimateLocalSurfacePoints(self, vid: int, nu: int, nv: int) -> np.ndarray:
        """Samples [nu * nv x 3] of the blended surface estimate around vertex vid."""
        out = np.zeros((nu * nv, 3), np.float32)
        check(_capi.lib().vsdmo_opt_estimate_surface_points(self.h, int(vid), int(nu), int(nv), _ptr(out), _capi.HOST))
        return out

    def feature_state(self):
        """(curves [nSurf x 12], fdeg [nSurf], flags [nSurf], (sector rowptr, table [nFeature x 20],
        surfaces [n x 16]) or None) of an optimiser with feature vertices, internal numbering."""
        nS, nF = self.mesh.info["nSurf"], self.mesh.info["nFeature"]
        curves = np.zeros((nS, 12), np.float32)
        fdeg = np.zeros(nS, np.int32)
        flags = np.zeros(nS, np.uint8)
        ns = C.c_int()
        check(_capi.lib().vsdmo_opt_feature_state(self.h, _ptr(curves), _ptr(fdeg), _ptr(flags), None, None, None,
                                                  C.byref(ns)))
        sectors = None
        if ns.value > 0:
            rp = np.zeros(nF + 1, np.int32)
            tab = np.zeros((nF, 20), np.int32)
            fs = np.zeros((ns.value, 16), np.float32)
            check(_capi.lib().vsdmo_opt_feature_state(self.h, None, None, None, _ptr(rp), _ptr(tab), _ptr(fs),
                                                      C.byref(ns)))
            sectors = (rp, tab, fs)
        return curves, fdeg, flags, sectors

    def surface_state(self):
        """(xyz_init [nSurf,3], local_surfaces [nSurf,16], nearest [nSurf]) of a surface
        optimiser, internal vertex numbering."""
        nS = self.mesh.info["nSurf"]
        x0 = np.zeros((nS, 3), np.float32)
        ls = np.zeros((nS, 16), np.float32)
        nn = np.zeros(nS, np.int32)
        check(_capi.lib().vsdmo_opt_surface_state(self.h, _ptr(x0), _ptr(ls), _ptr(nn)))
        return x0, ls, nn


class DMOTetClass(_DMOBase):
    """``DMO::DMOTetClass`` (``dmo/DMOTet.h:21-62``)."""

    def collect_pairs(self, n_iter: int, feats_dev_ptr: int, targets_dev_ptr: int, capacity: int) -> int:
        """Runs n_iter plain iterations, writing one (ring features, DMO displacement) pair per
        vertex update into caller-owned device arrays; returns the number of pairs."""
        n = C.c_long(0)
        check(_capi.lib().vsdmo_opt_collect_pairs(self.h, n_iter, C.c_void_p(feats_dev_ptr), C.c_void_p(targets_dev_ptr),
                                                  capacity, C.byref(n)))
        return n.value

    def set_model(self, model, reduced_n: int = 4, reduced_depth: int = 1, reduced_scale: float = 0.0175):
        """Learned mode: reduced grid around the model's proposal, plain search as fallback."""
        check(_capi.lib().vsdmo_opt_set_model(self.h, model.h if model is not None else None, reduced_n, reduced_depth,
                                              reduced_scale))
        self._model = model

    def set_proposal_schedule(self, once_after: int = -1):
        """Iterations (since the restart) from ``once_after`` on run the network once for all
        interior vertices from the positions at the iteration's start; earlier ones (all, with
        -1) run it before every colour class."""
        check(_capi.lib().vsdmo_opt_set_proposal_schedule(self.h, int(once_after)))

    def proposals(self, color: int) -> np.ndarray:
        """Network proposals [n x 3] of one colour class (fused inference kernel)."""
        r = self.mesh.array(A_COL_INNER)
        out = np.zeros((int(r[color + 1] - r[color]), 3), np.float32)
        check(_capi.lib().vsdmo_opt_proposals(self.h, color, _ptr(out)))
        return out

    def learned_counters(self):
        """(reduced accepted, fallbacks, fallbacks that moved, skipped by the active set)."""
        c = (C.c_ulonglong * 4)()
        check(_capi.lib().vsdmo_opt_learned_counters(self.h, c))
        return tuple(int(x) for x in c)


class ProposalModel:
    """The learned proposal network (no reference counterpart): 96 -> 128 -> 128 -> 128 -> 3."""

    def __init__(self, seed: int = 0, stream=None):
        self.h = C.c_void_p()
        check(_capi.lib().vsdmo_model_create(seed, C.c_void_p(stream), C.byref(self.h)))
        self.n_params = _capi.lib().vsdmo_model_num_params()

    def close(self):
        if getattr(self, "h", None):
            _capi.lib().vsdmo_model_destroy(self.h)
            self.h = None

    def __del__(self, _finalizing=sys.is_finalizing):
        # no library calls while the interpreter shuts down: the CUDA runtime may be gone
        # (bound as a default: module globals are cleared during shutdown)
        if _finalizing():
            return
        try:
            self.close()
        except Exception:
            pass

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.n_params, np.float32)
        check(_capi.lib().vsdmo_model_get_params(self.h, _ptr(p)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        check(_capi.lib().vsdmo_model_set_params(self.h, _ptr(p)))

    def forward(self, feats) -> np.ndarray:
        feats = np.ascontiguousarray(feats, np.float32)
        out = np.zeros((len(feats), 3), np.float32)
        check(_capi.lib().vsdmo_model_forward(self.h, _ptr(feats), len(feats), _ptr(out), _capi.HOST))
        return out

    def gradients(self, feats, targets):
        feats = np.ascontiguousarray(feats, np.float32)
        targets = np.ascontiguousarray(targets, np.float32)
        g = np.zeros(self.n_params, np.float32)
        loss = C.c_float(0)
        check(_capi.lib().vsdmo_model_gradients(self.h, _ptr(feats), _ptr(targets), len(feats), C.byref(loss), _ptr(g)))
        return float(loss.value), g

    def train(self, feats, targets, steps: int, batch: int = 4096, lr: float = 1e-3, seed: int = 0,
              device_ptrs=None, n_rows: int = 0):
        """Adam on minibatches drawn from (feats, targets); host arrays, or device pointers
        (device_ptrs = (feats_ptr, targets_ptr), n_rows). Returns the per-step loss."""
        hist = np.zeros(max(steps, 1), np.float32)
        if device_ptrs is not None:
            check(_capi.lib().vsdmo_model_train(self.h, C.c_void_p(device_ptrs[0]), C.c_void_p(device_ptrs[1]), n_rows,
                                                _capi.DEVICE, steps, batch, lr, seed, _ptr(hist)))
        else:
            feats = np.ascontiguousarray(feats, np.float32)
            targets = np.ascontiguousarray(targets, np.float32)
            check(_capi.lib().vsdmo_model_train(self.h, _ptr(feats), _ptr(targets), len(feats), _capi.HOST, steps, batch,
                                                lr, seed, _ptr(hist)))
        return hist[:steps]


def debug_gemm_bf16(A, B) -> np.ndarray:
    """D = bf16(A) . bf16(B)^T through the library's tensor-core GEMM (test entry point)."""
    A = np.ascontiguousarray(A, np.float32)
    B = np.ascontiguousarray(B, np.float32)
    D = np.zeros((A.shape[0], B.shape[0]), np.float32)
    check(_capi.lib().vsdmo_debug_gemm_bf16(_ptr(A), _ptr(B), A.shape[0], B.shape[0], A.shape[1], _ptr(D)))
    return D


def debug_set_wait_limit_ns(ns: int) -> None:
    """Test entry point: limit of the bounded device waits that report a timeout (batched
    colour-class waits, tensor-core GEMM and inference waits) on the current device; 0 makes
    them expire, a negative value restores the default of 1 s."""
    check(_capi.lib().vsdmo_debug_set_wait_limit_ns(int(ns)))


class DMOHexClass(_DMOBase):
    """``DMO::DMOHexClass`` (``dmo/DMOHex.h``): interior hex DMO with ``shapeMetricHex``."""


class DMOTriFlatClass(_DMOBase):
    """``DMO::DMOTriFlatClass`` (``dmo/DMOTriFlat.h:19-51``). The default criterion here is
    MEAN_RATIO; the reference's default argument, MIN_ANGLE (with ``fix_boundary=False`` for its
    sliding boundary), is passed explicitly."""
    _flat = 1


class DMOTriClass(_DMOBase):
    """``DMO::DMOTriClass`` (``dmo/DMOTri.h``): surface triangle DMO; feature vertices slide
    along their feature curves (``fix_boundary=True`` holds them)."""
    _flat = 0

    def __init__(self, dmo_mesh, qualityCriterium=QualityCriterium.MEAN_RATIO, gridScale: float = 0.5,
                 n_iter: int = 30, fix_boundary: bool = False, **kw):
        super().__init__(dmo_mesh, qualityCriterium, gridScale, n_iter, fix_boundary, **kw)


class DMOQuadClass(_DMOBase):
    """``DMO::DMOQuadClass`` (``dmo/DMOQuad.h``): surface quad DMO; feature vertices slide
    along their feature curves (``fix_boundary=True`` holds them)."""
    _flat = 0

    def __init__(self, dmo_mesh, qualityCriterium=QualityCriterium.MEAN_RATIO, gridScale: float = 0.5,
                 n_iter: int = 30, fix_boundary: bool = False, **kw):
        super().__init__(dmo_mesh, qualityCriterium, gridScale, n_iter, fix_boundary, **kw)


class DMOQuadFlatClass(_DMOBase):
    """Flat quad DMO: the 2D search of ``DMOTriFlatClass`` with the quad mean ratio against +z
    (``meanRatioMetricQuad(p, n)``, ``dmo/DMOQualityQuad.h:30-50``); the reference has no
    flat-quad class. ``grid_n`` 4 or 8."""
    _flat = 1


class BatchDMO:
    """Many independent flat tri / quad meshes optimised together (one persistent launch per
    iteration, replayed from a CUDA graph). ``meshes``: list of ``(elem_type, points [n x 3],
    elems [m x k])`` with mesh-local vertex ids, ``elem_type`` ``TRI`` or ``QUAD``. Stands in
    for a loop of ``DMOTriFlatClass`` objects, one per mesh."""

    def __init__(self, meshes, color_seed: int = 1, stream=None):
        types = np.array([int(t) for t, _, _ in meshes], np.int32)
        nv = np.array([len(p) for _, p, _ in meshes], np.int32)
        ne = np.array([len(e) for _, _, e in meshes], np.int32)
        xyz = np.ascontiguousarray(np.concatenate([np.asarray(p, np.float32).reshape(-1, 3) for _, p, _ in meshes]))
        el = np.ascontiguousarray(np.concatenate([np.asarray(e, np.int32).reshape(-1) for _, _, e in meshes]))
        self.n_meshes = len(meshes)
        self.n_vertices = int(nv.sum())
        self.elem_types, self.nv, self.ne = types, nv, ne
        h = C.c_void_p()
        check(_capi.lib().vsdmo_batch_create(len(meshes), _ptr(types), _ptr(nv), _ptr(ne), _ptr(xyz), _ptr(el),
                                              _capi.HOST, int(color_seed), C.c_void_p(stream), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            _capi.lib().vsdmo_batch_destroy(self.h)
            self.h = None

    def __del__(self, _finalizing=sys.is_finalizing):
        if _finalizing():
            return
        try:
            self.close()
        except Exception:
            pass

    def iterate(self, n: int = 1):
        check(_capi.lib().vsdmo_batch_iterate(self.h, int(n)))

    def iterate_async(self, n: int = 1):
        check(_capi.lib().vsdmo_batch_iterate_async(self.h, int(n)))

    def sync(self):
        check(_capi.lib().vsdmo_batch_sync(self.h))

    def restart(self):
        check(_capi.lib().vsdmo_batch_restart(self.h))

    def stats(self, iteration: int):
        """(min quality, mean quality, elements below the previous minimum) per mesh."""
        mn = np.zeros(self.n_meshes, np.float32)
        mean = np.zeros(self.n_meshes, np.float64)
        below = np.zeros(self.n_meshes, np.int32)
        check(_capi.lib().vsdmo_batch_stats(self.h, int(iteration), _ptr(mn), _ptr(mean), _ptr(below)))
        return mn, mean, below

    def positions(self) -> np.ndarray:
        out = np.zeros((self.n_vertices, 3), np.float32)
        check(_capi.lib().vsdmo_batch_get_positions(self.h, _ptr(out), _capi.HOST))
        return out

    def mesh_positions(self, i: int) -> np.ndarray:
        off = int(self.nv[:i].sum())
        return self.positions()[off:off + int(self.nv[i])]

    def set_positions(self, xyz):
        xyz = np.ascontiguousarray(xyz, np.float32)
        assert xyz.size == 3 * self.n_vertices
        check(_capi.lib().vsdmo_batch_set_positions(self.h, _ptr(xyz), _capi.HOST))

    def config(self):
        """(grid_n, depth, lanes) arrays, one entry per mesh."""
        n = np.zeros(self.n_meshes, np.int32)
        d = np.zeros(self.n_meshes, np.int32)
        l = np.zeros(self.n_meshes, np.int32)
        check(_capi.lib().vsdmo_batch_get_config(self.h, _ptr(n), _ptr(d), _ptr(l)))
        return n, d, l

    def set_config(self, grid_n, depth, lanes):
        b = lambda x: np.ascontiguousarray(np.broadcast_to(np.asarray(x, np.int32), (self.n_meshes,)))
        n, d, l = b(grid_n), b(depth), b(lanes)
        check(_capi.lib().vsdmo_batch_set_config(self.h, _ptr(n), _ptr(d), _ptr(l)))

    def autotune(self, probe_iters: int = 3) -> str:
        buf = C.create_string_buffer(4096)
        check(_capi.lib().vsdmo_batch_autotune(self.h, int(probe_iters), buf, len(buf)))
        return buf.value.decode()

    def info(self) -> dict:
        keys = ["meshes", "vertices", "items", "colors", "iterations", "blocks", "max_halfedges"]
        return {k: int(_capi.lib().vsdmo_batch_info(self.h, i)) for i, k in enumerate(keys)}

    def mesh_info(self, i: int) -> dict:
        out = np.zeros(8, np.int32)
        check(_capi.lib().vsdmo_batch_mesh_info(self.h, int(i), _ptr(out)))
        keys = ["v_off", "nV", "nE", "k", "colors", "free_begin", "free_end", "he_off"]
        return dict(zip(keys, (int(x) for x in out)))
