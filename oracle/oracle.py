"""ctypes wrapper of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loaded by tests/, ``__graft_entry__.smoke()`` and the CPU-baseline legs of ``bench.py``;
the product never imports this module. See ``vsdmo_oracle.h`` for what is restated and
from which reference lines.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

TRI, QUAD, TET, HEX = 0, 1, 2, 3
# color_seed value selecting the reference's JPL priorities n - i (OR_COLOR_REFERENCE); the flag
# COLOR_ROUNDS in a seed selects round colours (the reference's rule) with that seed's hashed
# priorities instead of the default smallest free colour (OR_COLOR_ROUNDS)
COLOR_REFERENCE = 0xFFFFFFFF
COLOR_ROUNDS = 0x80000000

A_XYZ, A_NEW_OF_OLD, A_ELEMS, A_SURF_TRIS, A_HE_ROWPTR, A_HALFEDGES, A_HF_ROWPTR, A_HALFFACES, \
    A_COL_FREE, A_COL_FEATURE, A_COL_INNER, A_IS_BOUNDARY1D, A_IS_FEATURE, A_IS_BOUNDARY2D, \
    A_FACE_NORMALS, A_VERTEX_NORMALS = range(16)
ARRAY_DTYPES = {A_XYZ: np.float32, A_FACE_NORMALS: np.float32, A_VERTEX_NORMALS: np.float32,
                A_IS_BOUNDARY1D: np.uint8, A_IS_FEATURE: np.uint8, A_IS_BOUNDARY2D: np.uint8}
ARRAY_NAMES = {A_XYZ: "xyz", A_NEW_OF_OLD: "new_of_old", A_ELEMS: "elems", A_SURF_TRIS: "surf_tris",
               A_HE_ROWPTR: "he_rowptr", A_HALFEDGES: "halfedges", A_HF_ROWPTR: "hf_rowptr",
               A_HALFFACES: "halffaces", A_COL_FREE: "col_free", A_COL_FEATURE: "col_feature",
               A_COL_INNER: "col_inner", A_IS_BOUNDARY1D: "is_boundary1d", A_IS_FEATURE: "is_feature",
               A_IS_BOUNDARY2D: "is_boundary2d", A_FACE_NORMALS: "face_normals",
               A_VERTEX_NORMALS: "vertex_normals"}
I_NAMES = ["nV", "nE", "nSurf", "nFeature", "nTris", "nHE", "nColorsFree", "nColorsFeature",
           "nColorsInner", "maxNumHalfedges", "maxNumTetrahedra", "isFlat"]

_lib = None


# where the reference's sources lie when they are present (this container; not the GPU box,
# which uses the builds under oracle/_ref/ that travel with the tree)
REF_SRC = os.environ.get("VSDMO_REFERENCE_SRC", "/root/reference/VSDMO/src")


def build():
    """The oracle library, and, where the reference's sources are present, the reference's own
    quality functions and mesh build / DMO as checkers (oracle/_ref/, Makefile target ``ref``)."""
    args = ["make", "-s", "-j8", "-C", HERE, "all"]
    if os.path.isdir(os.path.join(REF_SRC, "dmo")):
        args += ["ref-if-present", "REF=" + REF_SRC]
    subprocess.run(args, check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P, I, F, D, U = C.c_void_p, C.c_int, C.c_float, C.c_double, C.c_uint32
        L.or_mesh_build.restype = P
        L.or_mesh_build.argtypes = [I, I, P, I, P, U, C.c_char_p, I]
        L.or_mesh_free.argtypes = [P]
        L.or_mesh_info.argtypes = [P, I]
        L.or_mesh_array_len.restype = C.c_long
        L.or_mesh_array_len.argtypes = [P, I]
        L.or_mesh_array.argtypes = [P, I, P]
        L.or_color_jpl.argtypes = [I, P, P, U, P]
        L.or_priority.restype = U
        L.or_priority.argtypes = [U, U]
        for n in ("or_dmo_tet_f32", "or_dmo_tri2d_f32", "or_dmo_tet_ref32"):
            getattr(L, n).argtypes = [P, P, I, I, F, I]
        for n in ("or_dmo_tet_f64", "or_dmo_tri2d_f64"):
            getattr(L, n).argtypes = [P, P, I, I, D, P, I]
        L.or_element_qualities_f64.argtypes = [P, P, P]
        L.or_element_qualities_f32.argtypes = [P, P, P]
        L.or_optimize_f32.argtypes = [P, P, I, F, I, P, P]
        L.or_optimize_f64.argtypes = [P, P, I, D, I, P, P]
        L.or_surface_normals_f32.argtypes = [P, P, P, P]
        L.or_surface_normals_f64.argtypes = [P, P, P, P]
        L.or_surface_fit_f32.argtypes = [P, P, P, P]
        L.or_surface_fit_f64.argtypes = [P, P, P, P]
        L.or_surface_fit_ring_f32.argtypes = [P, P, P, P, I]
        L.or_surface_fit_ring_f64.argtypes = [P, P, P, P, I]
        L.or_update_nn_f32.argtypes = [P, P, P, P]
        L.or_update_nn_f64.argtypes = [P, P, P, P]
        L.or_dmo_surf_f32.argtypes = [P, P, P, P, P, P, I, I, F, I]
        L.or_dmo_surf_f64.argtypes = [P, P, P, P, P, P, I, I, D, P, I]
        L.or_surface_qualities_f32.argtypes = [P, P, P]
        L.or_surface_qualities_f64.argtypes = [P, P, P]
        L.or_optimize_surf_f32.argtypes = [P, P, I, F, I, P, P]
        L.or_optimize_surf_f64.argtypes = [P, P, I, D, I, P, P]
        L.or_dmo_flat_f32.argtypes = [P, P, I, I, F, I, I, I]
        L.or_dmo_quad2d_f64.argtypes = [P, P, I, I, D, P, I]
        L.or_q_quad2d_f32.restype = F
        L.or_q_quad2d_f32.argtypes = [P, P, P, P]
        L.or_dmo_hex_f32.argtypes = [P, P, I, I, F, I]
        L.or_dmo_hex_f64.argtypes = [P, P, I, I, D, P, I]
        L.or_hex_qualities_f32.argtypes = [P, P, P]
        L.or_hex_qualities_f64.argtypes = [P, P, P]
        L.or_optimize_hex_f32.argtypes = [P, P, I, F, I, P, P]
        L.or_optimize_hex_f64.argtypes = [P, P, I, D, I, P, P]
        L.or_dmo_angle_f64.argtypes = [P, P, I, I, D, I, P, I]
        L.or_surface_points_f32.argtypes = [P, P, P, P, P, I, I, I, F, I, P]
        L.or_feature_flags.argtypes = [P, P, P, P]
        L.or_feature_surfaces_f32.restype = I
        L.or_feature_surfaces_f32.argtypes = [P, P, P, P, P, P, I]
        L.or_feature_surfaces_f64.restype = I
        L.or_feature_surfaces_f64.argtypes = [P, P, P, P, P, P, I]
        L.or_dmo_surf_feat_f32.argtypes = [P, P, P, P, P, P, P, P, P, I, I, F, I]
        L.or_dmo_vol_surf_f32.argtypes = [P, P, P, P, P, P, P, P, I, I, F, I]
        L.or_dmo_vol_surf_f64.argtypes = [P, P, P, P, P, P, P, P, I, I, D, P, I]
        L.or_dmo_surf_feat_f64.argtypes = [P, P, P, P, P, P, P, P, P, I, I, D, P, I]
        L.or_surface_fit_1d_f32.argtypes = [P, P, P, P]
        L.or_surface_fit_1d_f64.argtypes = [P, P, P, P]
        L.or_dmo_1d_f32.argtypes = [P, P, P, P, P, P, P, P, I, I, F, I]
        L.or_dmo_1d_f64.argtypes = [P, P, P, P, P, P, P, P, I, I, D, P, I]
        L.or_angle_qualities_f64.argtypes = [P, P, I, P]
        L.or_dmo_tet_learned_f32.argtypes = [P, P, I, I, P, I, F, I, I, F, P, I]
        L.or_dmo_hex_cond_f32.argtypes = [P, P, I, I, F, I]
        L.or_dmo_hex_cond_f64.argtypes = [P, P, I, I, D, P, I]
        L.or_hex_cond_qualities_f32.argtypes = [P, P, P]
        L.or_hex_cond_qualities_f64.argtypes = [P, P, P]
        L.or_set_criterion.argtypes = [I]
        L.or_set_criterion.restype = None
        for n in ("or_q_tet_min_angle_f64", "or_q_tet_max_angle_f64"):
            getattr(L, n).restype = D
            getattr(L, n).argtypes = [P, P, P, P]
        for n in ("or_q_tri2d_min_angle_f64", "or_q_tri2d_max_angle_f64"):
            getattr(L, n).restype = D
            getattr(L, n).argtypes = [P, P, P]
        L.or_q_tet_mean_ratio_f64.restype = D
        L.or_q_tet_mean_ratio_f64.argtypes = [P, P, P, P]
        L.or_q_tet_mean_ratio_f32.restype = F
        L.or_q_tet_mean_ratio_f32.argtypes = [P, P, P, P]
        L.or_q_tri2d_mean_ratio_f64.restype = D
        L.or_q_tri2d_mean_ratio_f64.argtypes = [P, P, P]
        L.or_q_tri2d_mean_ratio_f32.restype = F
        L.or_q_tri2d_mean_ratio_f32.argtypes = [P, P, P]
        L.or_q_hex_f64.restype = D
        L.or_q_hex_f64.argtypes = [P]
        L.or_q_tri3d_f64.restype = D
        L.or_q_tri3d_f64.argtypes = [P, P, P]
        L.or_q_tri3d_angle_f64.restype = D
        L.or_q_tri3d_angle_f64.argtypes = [P, P, P, P, I]
        L.or_q_quad_f64.restype = D
        L.or_q_quad_f64.argtypes = [P, P, P, P, P]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class OracleMesh:
    """Connectivity, colouring and DMO of the reference, on the CPU."""

    def __init__(self, elem_type, xyz, elems, color_seed=1):
        xyz = np.ascontiguousarray(xyz, dtype=np.float32)
        elems = np.ascontiguousarray(elems, dtype=np.int32)
        err = C.create_string_buffer(512)
        self.h = lib().or_mesh_build(elem_type, len(xyz), _p(xyz), len(elems), _p(elems),
                                     color_seed, err, 512)
        if not self.h:
            raise ValueError("oracle mesh build failed: " + err.value.decode())
        self.elem_type = elem_type
        self.info = {n: lib().or_mesh_info(self.h, i) for i, n in enumerate(I_NAMES)}

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_mesh_free(self.h)
            self.h = None

    def array(self, aid):
        n = lib().or_mesh_array_len(self.h, aid)
        out = np.zeros(max(n, 0), dtype=ARRAY_DTYPES.get(aid, np.int32))
        if n > 0:
            lib().or_mesh_array(self.h, aid, _p(out))
        return out

    def arrays(self):
        return {ARRAY_NAMES[a]: self.array(a) for a in ARRAY_NAMES}

    @property
    def xyz(self):
        return self.array(A_XYZ).reshape(-1, 3)

    def color_ranges(self):
        """(pass, start, end) of every colour class in doIteration order."""
        if self.elem_type in (TET, HEX):
            off = self.array(A_COL_INNER)
        else:
            off = self.array(A_COL_FREE)
        return [(int(off[c]), int(off[c + 1])) for c in range(len(off) - 1)]

    # ---- DMO steps ----------------------------------------------------------------------
    def dmo_color_f32(self, xyz, v0, v1, grid_scale=0.5, nthreads=0):
        xyz = np.ascontiguousarray(xyz, dtype=np.float32).copy()
        fn = {TET: lib().or_dmo_tet_f32, HEX: lib().or_dmo_hex_f32}.get(self.elem_type, lib().or_dmo_tri2d_f32)
        fn(self.h, _p(xyz), v0, v1, grid_scale, nthreads)
        return xyz

    def dmo_hex_cond_f32(self, xyz, v0, v1, grid_scale=0.5, nthreads=0):
        """One colour class of interior hex vertices under the condition-number quality (f32)."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float32).copy()
        lib().or_dmo_hex_cond_f32(self.h, _p(xyz), v0, v1, grid_scale, nthreads)
        return xyz

    def dmo_hex_cond_f64(self, xyz, v0, v1, grid_scale=0.5, nthreads=0):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).copy()
        margin = np.zeros(max(v1 - v0, 1))
        lib().or_dmo_hex_cond_f64(self.h, _p(xyz), v0, v1, grid_scale, _p(margin), nthreads)
        return xyz, margin[: v1 - v0]

    def hex_cond_qualities(self, xyz, dtype=np.float64):
        xyz = np.ascontiguousarray(xyz, dtype=dtype)
        q = np.zeros(self.info["nE"], dtype=dtype)
        fn = lib().or_hex_cond_qualities_f64 if dtype == np.float64 else lib().or_hex_cond_qualities_f32
        fn(self.h, _p(xyz), _p(q))
        return q

    def dmo_tet_learned_f32(self, xyz, v0, v1, Y, rn=4, rdepth=2, rscale=0.012, grid_scale=0.5, nthreads=0):
        """Learned mode, one colour class: (positions, queued mask of the plain-search fallbacks)."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float32).copy()
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        queued = np.zeros(max(v1 - v0, 1), np.uint8)
        lib().or_dmo_tet_learned_f32(self.h, _p(xyz), v0, v1, _p(Y), Y.shape[1], grid_scale, rn, rdepth, rscale,
                                     _p(queued), nthreads)
        return xyz, queued[: v1 - v0].astype(bool)

    def dmo_flat_f32(self, xyz, v0, v1, nq=8, depth=3, grid_scale=0.5, nthreads=0):
        """Flat tri / quad colour class with an nq x nq grid and `depth` levels (batched optimiser)."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float32).copy()
        lib().or_dmo_flat_f32(self.h, _p(xyz), v0, v1, grid_scale, nq, depth, nthreads)
        return xyz

    def dmo_quad2d_f64(self, xyz, v0, v1, grid_scale=0.5, nthreads=0):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).copy()
        margin = np.zeros(max(v1 - v0, 1), dtype=np.float64)
        lib().or_dmo_quad2d_f64(self.h, _p(xyz), v0, v1, grid_scale, _p(margin), nthreads)
        return xyz, margin[: v1 - v0]

    def dmo_angle_f64(self, xyz, v0, v1, max_angle=False, grid_scale=0.5, nthreads=0):
        """One colour class with the MIN_ANGLE (or MAX_ANGLE) criterion, literal in double."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).copy()
        margin = np.zeros(max(v1 - v0, 1), dtype=np.float64)
        lib().or_dmo_angle_f64(self.h, _p(xyz), v0, v1, grid_scale, int(max_angle), _p(margin), nthreads)
        return xyz, margin[: v1 - v0]

    def surface_points_f32(self, xyz, state, vid, nu, nv, estimate, grid_scale=0.5):
        """Sample grid of a surface view; state = (xyz_init, local_surfaces, nearest)."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float32)
        x0, ls, nn = (np.ascontiguousarray(a) for a in state)
        out = np.zeros((nu * nv, 3), np.float32)
        lib().or_surface_points_f32(self.h, _p(xyz), _p(x0), _p(ls), _p(nn), int(vid), int(nu), int(nv), grid_scale,
                                    int(estimate), _p(out))
        return out

    # ---- 1D feature / boundary pass ---------------------------------------------------------
    def feature_flags(self, xyz):
        """(fdeg [nSurf], opt [nSurf] uint8) from the positions."""
        nS = self.info["nSurf"]
        fdeg = np.zeros(nS, np.int32)
        opt = np.zeros(nS, np.uint8)
        lib().or_feature_flags(self.h, _p(np.ascontiguousarray(xyz, np.float32)), _p(fdeg), _p(opt))
        return fdeg, opt

    def sector_surfaces(self, xyz, fn, dtype=np.float32):
        """Per-sector surfaces of the feature vertices: (rowptr [nFeature+1], table
        [nFeature x 20], surfaces [nSectors x 16]); fn: face normals [nTris x 3]."""
        nF = self.info["nFeature"]
        cap = 20 * max(nF, 1)
        rowptr = np.zeros(nF + 1, np.int32)
        table = np.zeros(max(nF, 1) * 20, np.int32)
        ls = np.zeros((cap, 16), dtype)
        fn_ = lib().or_feature_surfaces_f32 if dtype == np.float32 else lib().or_feature_surfaces_f64
        ns = fn_(self.h, _p(np.ascontiguousarray(xyz, dtype)), _p(np.ascontiguousarray(fn, dtype)), _p(rowptr),
                 _p(table), _p(ls), cap)
        if ns < 0:
            raise ValueError("feature vertex beyond the sector table sizes")
        return rowptr, table[: 20 * nF].reshape(nF, 20), ls[:ns]

    def dmo_surf_feat_f32(self, xyz, x0, ls, nn, vn, sectors, v0, v1, grid_scale=0.5, nthreads=0):
        xyz = np.ascontiguousarray(xyz, dtype=np.float32).copy()
        rp, tab, fs = (np.ascontiguousarray(a) for a in sectors)
        lib().or_dmo_surf_feat_f32(self.h, _p(xyz), _p(np.ascontiguousarray(x0, np.float32)),
                                   _p(np.ascontiguousarray(ls, np.float32)), _p(np.ascontiguousarray(nn, np.int32)),
                                   _p(np.ascontiguousarray(vn, np.float32)), _p(rp), _p(tab),
                                   _p(np.ascontiguousarray(fs, np.float32)), v0, v1, grid_scale, nthreads)
        return xyz

    def dmo_surf_feat_f64(self, xyz, x0, ls, nn, vn, sectors, v0, v1, grid_scale=0.5, nthreads=0):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).copy()
        rp, tab, fs = sectors
        margin = np.zeros(max(v1 - v0, 1))
        lib().or_dmo_surf_feat_f64(self.h, _p(xyz), _p(np.ascontiguousarray(x0, np.float64)),
                                   _p(np.ascontiguousarray(ls, np.float64)), _p(np.ascontiguousarray(nn, np.int32)),
                                   _p(np.ascontiguousarray(vn, np.float64)), _p(np.ascontiguousarray(rp, np.int32)),
                                   _p(np.ascontiguousarray(tab, np.int32)), _p(np.ascontiguousarray(fs, np.float64)),
                                   v0, v1, grid_scale, _p(margin), nthreads)
        return xyz, margin[: v1 - v0]

    def dmo_vol_surf_f32(self, xyz, x0, ls, nn, sectors, v0, v1, grid_scale=0.5, nthreads=0):
        """Boundary-surface pass of a tet or hex mesh over the free boundary class [v0, v1)."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float32).copy()
        rp, tab, fs = (None, None, None) if sectors is None else (np.ascontiguousarray(a) for a in sectors)
        lib().or_dmo_vol_surf_f32(self.h, _p(xyz), _p(np.ascontiguousarray(x0, np.float32)),
                                  _p(np.ascontiguousarray(ls, np.float32)), _p(np.ascontiguousarray(nn, np.int32)),
                                  None if rp is None else _p(rp), None if tab is None else _p(tab),
                                  None if fs is None else _p(np.ascontiguousarray(fs, np.float32)), v0, v1,
                                  grid_scale, nthreads)
        return xyz

    def dmo_vol_surf_f64(self, xyz, x0, ls, nn, sectors, v0, v1, grid_scale=0.5, nthreads=0):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).copy()
        margin = np.zeros(max(v1 - v0, 1))
        a = [None, None, None] if sectors is None else [np.ascontiguousarray(sectors[0], np.int32),
                                                       np.ascontiguousarray(sectors[1], np.int32),
                                                       np.ascontiguousarray(sectors[2], np.float64)]
        lib().or_dmo_vol_surf_f64(self.h, _p(xyz), _p(np.ascontiguousarray(x0, np.float64)),
                                  _p(np.ascontiguousarray(ls, np.float64)), _p(np.ascontiguousarray(nn, np.int32)),
                                  *[None if x is None else _p(x) for x in a], v0, v1, grid_scale, _p(margin), nthreads)
        return xyz, margin[: v1 - v0]

    def curves_f32(self, xyz, vn):
        nS = self.info["nSurf"]
        out = np.zeros((nS, 12), np.float32)
        lib().or_surface_fit_1d_f32(self.h, _p(np.ascontiguousarray(xyz, np.float32)),
                                    _p(np.ascontiguousarray(vn, np.float32)), _p(out))
        return out

    def curves_f64(self, xyz, vn):
        nS = self.info["nSurf"]
        out = np.zeros((nS, 12), np.float64)
        lib().or_surface_fit_1d_f64(self.h, _p(np.ascontiguousarray(xyz, np.float64)),
                                    _p(np.ascontiguousarray(vn, np.float64)), _p(out))
        return out

    def dmo_1d_f32(self, xyz, x0, curves, nn, vn, fdeg, opt, v0, v1, grid_scale=0.5, nthreads=0):
        xyz = np.ascontiguousarray(xyz, dtype=np.float32).copy()
        a = [np.ascontiguousarray(x) for x in (x0, curves, nn, vn, fdeg, opt)]
        lib().or_dmo_1d_f32(self.h, _p(xyz), *[_p(x) for x in a], v0, v1, grid_scale, nthreads)
        return xyz

    def dmo_1d_f64(self, xyz, x0, curves, nn, vn, fdeg, opt, v0, v1, grid_scale=0.5, nthreads=0):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).copy()
        a = [np.ascontiguousarray(x0, np.float64), np.ascontiguousarray(curves, np.float64),
             np.ascontiguousarray(nn, np.int32), np.ascontiguousarray(vn, np.float64),
             np.ascontiguousarray(fdeg, np.int32), np.ascontiguousarray(opt, np.uint8)]
        margin = np.zeros(max(v1 - v0, 1), np.float64)
        lib().or_dmo_1d_f64(self.h, _p(xyz), *[_p(x) for x in a], v0, v1, grid_scale, _p(margin), nthreads)
        return xyz, margin[: v1 - v0]

    def angle_qualities_f64(self, xyz, max_angle=False):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        q = np.zeros(self.info["nE"], dtype=np.float64)
        lib().or_angle_qualities_f64(self.h, _p(xyz), int(max_angle), _p(q))
        return q

    def dmo_color_ref32(self, xyz, v0, v1, grid_scale=0.5, nthreads=0):
        """The reference kernel's own float arithmetic (tet interior only)."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float32).copy()
        lib().or_dmo_tet_ref32(self.h, _p(xyz), v0, v1, grid_scale, nthreads)
        return xyz

    def dmo_color_f64(self, xyz, v0, v1, grid_scale=0.5, nthreads=0):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).copy()
        margin = np.zeros(max(v1 - v0, 1), dtype=np.float64)
        fn = {TET: lib().or_dmo_tet_f64, HEX: lib().or_dmo_hex_f64}.get(self.elem_type, lib().or_dmo_tri2d_f64)
        fn(self.h, _p(xyz), v0, v1, grid_scale, _p(margin), nthreads)
        return xyz, margin[: v1 - v0]

    @property
    def is_surface(self):
        """tri mesh that is not flat, or a quad mesh: optimised by the surface kernels"""
        return self.elem_type == QUAD or (self.elem_type == TRI and not self.info["isFlat"])

    def optimize_f32(self, xyz, n_iter, grid_scale=0.5, nthreads=0):
        xyz = np.ascontiguousarray(xyz, dtype=np.float32).copy()
        mn = np.zeros(n_iter); mean = np.zeros(n_iter)
        fn = lib().or_optimize_surf_f32 if self.is_surface else lib().or_optimize_f32
        if self.elem_type == HEX:
            fn = lib().or_optimize_hex_f32
        fn(self.h, _p(xyz), n_iter, grid_scale, nthreads, _p(mn), _p(mean))
        return xyz, mn, mean

    def optimize_f64(self, xyz, n_iter, grid_scale=0.5, nthreads=0):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).copy()
        mn = np.zeros(n_iter); mean = np.zeros(n_iter)
        fn = lib().or_optimize_surf_f64 if self.is_surface else lib().or_optimize_f64
        if self.elem_type == HEX:
            fn = lib().or_optimize_hex_f64
        fn(self.h, _p(xyz), n_iter, grid_scale, nthreads, _p(mn), _p(mean))
        return xyz, mn, mean

    # ---- surface state (quadric fit, nearest initial vertex, normals) --------------------
    def surface_state_f32(self, xyz, ring=1):
        """(xyz_init, local_surfaces[nSurf,16], nearest[nSurf], face_normals, vertex_normals)"""
        xyz = np.ascontiguousarray(xyz, dtype=np.float32)
        nS, nF = self.info["nSurf"], self.info["nTris"]
        fn = np.zeros((nF, 3), np.float32); vn = np.zeros((nS, 3), np.float32)
        lib().or_surface_normals_f32(self.h, _p(xyz), _p(fn), _p(vn))
        ls = np.zeros((nS, 16), np.float32)
        lib().or_surface_fit_ring_f32(self.h, _p(xyz), _p(vn), _p(ls), int(ring))
        return xyz.copy(), ls, np.arange(nS, dtype=np.int32), fn, vn

    def surface_normals_f64(self, xyz):
        """(face normals [nTris, 3], vertex normals [nSurf, 3]) in double."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        fn = np.zeros((self.info["nTris"], 3)); vn = np.zeros((self.info["nSurf"], 3))
        lib().or_surface_normals_f64(self.h, _p(xyz), _p(fn), _p(vn))
        return fn, vn

    def optimize_surf_features_f64(self, xyz, n_iter, grid_scale=0.5, nthreads=0):
        """DMOTriClass / DMOQuadClass::doIteration (dmo/DMOTri.cu:128-165, dmo/DMOQuad.cu:125-162)
        in double for a surface with feature vertices: free colours on their local (or sector)
        surfaces, then the feature colours along their curves, the nearest-initial-vertex walk and
        new normals; the quadric, sector and curve fits from the initial positions. Returns
        (positions, per-iteration minimum, per-iteration mean)."""
        x32 = np.ascontiguousarray(xyz, np.float32)
        x = x32.astype(np.float64)
        x0, ls, nn, vn = self.surface_state_f64(x32)
        fn, vn = self.surface_normals_f64(x)
        feat = self.info["nFeature"] > 0
        sectors = self.sector_surfaces(x32, fn, dtype=np.float64) if feat else None
        fdeg, flags = self.feature_flags(x32)
        curves = self.curves_f64(x32, vn)
        free = self.array(A_COL_FREE)
        cf = self.array(A_COL_FEATURE)
        mn, mean = [], []
        for _ in range(n_iter):
            for c in range(len(free) - 1):
                v0, v1 = int(free[c]), int(free[c + 1])
                if feat:
                    x, _ = self.dmo_surf_feat_f64(x, x0, ls, nn, vn, sectors, v0, v1, grid_scale, nthreads)
                else:
                    x, _ = self.dmo_surf_color_f64(x, x0, ls, nn, vn, v0, v1, grid_scale, nthreads)
            for c in range(len(cf) - 1):
                x, _ = self.dmo_1d_f64(x, x0, curves, nn, vn, fdeg, flags, int(cf[c]), int(cf[c + 1]),
                                       grid_scale, nthreads)
            nn = nn.copy()
            lib().or_update_nn_f64(self.h, _p(x), _p(x0), _p(nn))
            fn, vn = self.surface_normals_f64(x)
            q = self.element_qualities_f64(x)
            mn.append(float(q.min())); mean.append(float(q.mean()))
        return x, np.array(mn), np.array(mean)

    def surface_state_f64(self, xyz, ring=1):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        nS = self.info["nSurf"]
        vn = self.array(A_VERTEX_NORMALS).reshape(-1, 3).astype(np.float64)
        ls = np.zeros((nS, 16), np.float64)
        lib().or_surface_fit_ring_f64(self.h, _p(xyz), _p(vn), _p(ls), int(ring))
        return xyz.copy(), ls, np.arange(nS, dtype=np.int32), vn

    def dmo_surf_color_f32(self, xyz, state, v0, v1, grid_scale=0.5, nthreads=0):
        x0, ls, nn, _, vn = state
        xyz = np.ascontiguousarray(xyz, dtype=np.float32).copy()
        lib().or_dmo_surf_f32(self.h, _p(xyz), _p(x0), _p(ls), _p(nn), _p(vn), v0, v1, grid_scale, nthreads)
        return xyz

    def dmo_surf_color_f64(self, xyz, x0, ls, nn, vn, v0, v1, grid_scale=0.5, nthreads=0):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).copy()
        margin = np.zeros(max(v1 - v0, 1))
        lib().or_dmo_surf_f64(self.h, _p(xyz), _p(np.ascontiguousarray(x0, np.float64)),
                              _p(np.ascontiguousarray(ls, np.float64)), _p(np.ascontiguousarray(nn, np.int32)),
                              _p(np.ascontiguousarray(vn, np.float64)), v0, v1, grid_scale, _p(margin), nthreads)
        return xyz, margin[: v1 - v0]

    def element_qualities_f64(self, xyz):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        q = np.zeros(self.info["nE"], dtype=np.float64)
        fn = lib().or_surface_qualities_f64 if self.is_surface else lib().or_element_qualities_f64
        if self.elem_type == HEX:
            fn = lib().or_hex_qualities_f64
        fn(self.h, _p(xyz), _p(q))
        return q

    def element_qualities_f32(self, xyz):
        xyz = np.ascontiguousarray(xyz, dtype=np.float32)
        q = np.zeros(self.info["nE"], dtype=np.float32)
        fn = lib().or_surface_qualities_f32 if self.is_surface else lib().or_element_qualities_f32
        if self.elem_type == HEX:
            fn = lib().or_hex_qualities_f32
        fn(self.h, _p(xyz), _p(q))
        return q


MEAN_RATIO, MIN_ANGLE, MAX_ANGLE, CONDITION = 0, 4, 6, 7


class criterion:
    """Context manager: the criterion of the f64 surface, 1D and boundary restatements and of
    the surface element qualities (process-wide oracle state; mean ratio outside the block)."""

    def __init__(self, c):
        self.c = int(c)

    def __enter__(self):
        lib().or_set_criterion(self.c)
        return self

    def __exit__(self, *exc):
        lib().or_set_criterion(MEAN_RATIO)
        return False


def color_jpl(rowptr, col, seed=1):
    rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
    col = np.ascontiguousarray(col, dtype=np.int32)
    n = len(rowptr) - 1
    colors = np.zeros(n, dtype=np.int32)
    nc = lib().or_color_jpl(n, _p(rowptr), _p(col), seed, _p(colors))
    return colors, nc


def q_tet(p, dtype=np.float64):
    p = [np.ascontiguousarray(x, dtype=dtype) for x in p]
    f = lib().or_q_tet_mean_ratio_f64 if dtype == np.float64 else lib().or_q_tet_mean_ratio_f32
    return f(*[_p(x) for x in p])


def q_tri2d(p, dtype=np.float64):
    p = [np.ascontiguousarray(x, dtype=dtype) for x in p]
    f = lib().or_q_tri2d_mean_ratio_f64 if dtype == np.float64 else lib().or_q_tri2d_mean_ratio_f32
    return f(*[_p(x) for x in p])


# ---- the reference's own element quality functions (oracle/_ref/libref_quality.so) ----------
# Built by ``make ref`` from the reference's dmo/DMOQuality.h as it lies (ref_quality.cu); they
# run on the GPU. Item kinds (ref_quality.cu RefFn) and the reference's QualityCriterium values:
RQ_TET, RQ_HEX, RQ_QUAD, RQ_TRI, RQ_TRI2D, RQ_TRI_N, RQ_QUAD_N = range(7)
REF_MEAN_RATIO, REF_MIN_ANGLE, REF_MAX_ANGLE = 0, 4, 6
REF_LIB_PATH = os.path.join(HERE, "_ref", "libref_quality.so")
_ref = None


def ref_lib():
    """The compiled reference quality functions, or None where they were not built (the
    reference sources were absent when ``build()`` ran)."""
    global _ref
    if _ref is None and os.path.exists(REF_LIB_PATH):
        L = C.CDLL(REF_LIB_PATH)
        L.refq_eval.restype = C.c_int
        L.refq_eval.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
        _ref = L
    return _ref


def ref_quality(fn, crit, pts, nrm=None):
    """The reference function ``fn`` (RQ_*) with criterion ``crit`` on each item: pts has shape
    (n, corners, 3), nrm (n, 3) for RQ_TRI_N / RQ_QUAD_N. Float32 results from the GPU."""
    pts = np.ascontiguousarray(pts, dtype=np.float32)
    n = pts.shape[0]
    out = np.zeros(n, dtype=np.float32)
    nr = None if nrm is None else np.ascontiguousarray(nrm, dtype=np.float32)
    st = ref_lib().refq_eval(fn, crit, _p(pts), None if nr is None else _p(nr), n, _p(out))
    if st != 0:
        raise RuntimeError(f"refq_eval failed with CUDA error {st}")
    return out


def element_metric_f64(fn, crit, pts, nrm=None):
    """The oracle's FP64 restatement of the same reference function on each item (the
    functions the oracle's DMO and quality restatements use)."""
    L = lib()
    pts = np.ascontiguousarray(pts, dtype=np.float64)
    nrm = None if nrm is None else np.ascontiguousarray(nrm, dtype=np.float64)
    out = np.zeros(pts.shape[0])
    for i, e in enumerate(pts):
        c = [_p(e[j]) for j in range(e.shape[0])]
        if fn == RQ_TET:
            f = {REF_MEAN_RATIO: L.or_q_tet_mean_ratio_f64, REF_MIN_ANGLE: L.or_q_tet_min_angle_f64,
                 REF_MAX_ANGLE: L.or_q_tet_max_angle_f64}[crit]
            out[i] = f(*c)
        elif fn == RQ_HEX:
            out[i] = L.or_q_hex_f64(_p(e))
        elif fn == RQ_QUAD:
            out[i] = L.or_q_quad_f64(*c, None)
        elif fn == RQ_QUAD_N:
            out[i] = L.or_q_quad_f64(*c, _p(nrm[i]))
        elif fn == RQ_TRI2D:
            f = {REF_MEAN_RATIO: L.or_q_tri2d_mean_ratio_f64, REF_MIN_ANGLE: L.or_q_tri2d_min_angle_f64,
                 REF_MAX_ANGLE: L.or_q_tri2d_max_angle_f64}[crit]
            out[i] = f(*c)
        elif fn in (RQ_TRI, RQ_TRI_N):
            nv = None if fn == RQ_TRI else _p(nrm[i])
            if crit == REF_MEAN_RATIO:
                q = L.or_q_tri3d_f64(*c)
                if fn == RQ_TRI_N:
                    t = np.cross(e[1] - e[0], e[2] - e[0])
                    d = float(np.dot(t / np.linalg.norm(t), nrm[i]))
                    q = q if d > 0 else (-q if d < 0 else 0.0)
                out[i] = q
            else:
                out[i] = L.or_q_tri3d_angle_f64(*c, nv, int(crit == REF_MAX_ANGLE))
        else:
            raise ValueError(fn)
    return out


# ---- the reference's own mesh build and DMO (oracle/_ref/libref_vsdmo.so) --------------------
# Built by ``make ref`` from the reference's mesh/ and dmo/ sources as they lie (ref_vsdmo.cu,
# ref_prelude_vsdmo.h); it runs on the GPU. Colouring: the reference's color_jpl (priorities
# n - i) stands in for its closed cusparseScsrcolor, unless COLOURING_CUSPARSE (the closed one),
# COLOURING_HASHED (the reference's JPL rounds with the library's hashed priorities) or
# COLOURING_FIRST_FIT (the library's default colouring of those priorities) is asked.
REFVS_LIB_PATH = os.path.join(HERE, "_ref", "libref_vsdmo.so")
COLOURING_JPL, COLOURING_CUSPARSE, COLOURING_HASHED, COLOURING_FIRST_FIT = 0, 1, 2, 3
_refvs = None


def refvs_lib():
    """The reference's compiled mesh build and DMO, or None where they were not built."""
    global _refvs
    if _refvs is None and os.path.exists(REFVS_LIB_PATH):
        L = C.CDLL(REFVS_LIB_PATH)
        P, I, F = C.c_void_p, C.c_int, C.c_float
        L.refvs_set_colouring.argtypes = [I, C.c_uint32]
        L.refvs_set_colouring.restype = None
        L.refvs_mesh_create.argtypes = [I, P, I, P, I]
        L.refvs_mesh_create.restype = P
        L.refvs_mesh_destroy.argtypes = [P]
        L.refvs_mesh_destroy.restype = None
        L.refvs_mesh_info.argtypes = [P, I]
        L.refvs_mesh_info.restype = I
        L.refvs_mesh_array.argtypes = [P, I, P]
        L.refvs_mesh_array.restype = C.c_long
        L.refvs_set_positions.argtypes = [P, P]
        L.refvs_set_positions.restype = None
        L.refvs_colour_launch.argtypes = [P, I, F]
        L.refvs_colour_sweeps.argtypes = [P, I, F, C.POINTER(F)]
        L.refvs_opt_create.argtypes = [P, I, F, I]
        L.refvs_opt_iterate.argtypes = [P, I]
        L.refvs_opt_quality.argtypes = [P]
        L.refvs_opt_quality.restype = F
        L.refvs_opt_element_qualities.argtypes = [P, P]
        L.refvs_opt_surface_state.argtypes = [P, P, P, P]
        L.refvs_opt_surface_colour.argtypes = [P, I]
        _refvs = L
    return _refvs


class RefMesh:
    """A mesh built by the reference's own code (MeshXxxGPU::init + DMOMeshXxx) on the GPU, with
    its interior / flat colour launches and its optimiser classes. Arrays, info items and the
    internal vertex order are in the library's formats (VSDMO_A_*)."""

    def __init__(self, kind, xyz, elems, colouring=COLOURING_JPL, color_seed=1):
        L = refvs_lib()
        L.refvs_set_colouring(int(colouring), int(color_seed))
        xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
        k = {TRI: 3, QUAD: 4, TET: 4, HEX: 8}[kind]
        el = np.ascontiguousarray(elems, dtype=np.int32).reshape(-1, k)
        self.kind, self.k = kind, k
        self.h = L.refvs_mesh_create(kind, _p(xyz), len(xyz), _p(el), len(el))
        L.refvs_set_colouring(COLOURING_JPL, 1)
        if not self.h:
            raise RuntimeError("the reference did not build the mesh")
        self.info = {n: L.refvs_mesh_info(self.h, i) for i, n in enumerate(I_NAMES)}

    def close(self):
        if self.h:
            refvs_lib().refvs_mesh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def array(self, aid):
        L = refvs_lib()
        n = L.refvs_mesh_array(self.h, aid, None)
        if n < 0:
            return None
        a = np.zeros(max(n, 0), dtype=ARRAY_DTYPES.get(aid, np.int32))
        if n > 0:
            L.refvs_mesh_array(self.h, aid, _p(a))
        return a

    def arrays(self):
        out = {}
        for aid in ARRAY_NAMES:
            if aid == A_NEW_OF_OLD:
                continue
            a = self.array(aid)
            if a is not None:
                out[ARRAY_NAMES[aid]] = a
        return out

    def positions(self):
        return self.array(A_XYZ).reshape(-1, 3)

    def set_positions(self, xyz):
        xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
        refvs_lib().refvs_set_positions(self.h, _p(xyz))

    def colour_launch(self, cid, grid_scale=0.5):
        st = refvs_lib().refvs_colour_launch(self.h, int(cid), float(grid_scale))
        if st != 0:
            raise RuntimeError(f"reference colour launch failed ({st})")

    def colour_sweeps(self, n_iter, grid_scale=0.5):
        ms = C.c_float(0)
        st = refvs_lib().refvs_colour_sweeps(self.h, int(n_iter), float(grid_scale), C.byref(ms))
        if st != 0:
            raise RuntimeError(f"reference colour sweeps failed ({st})")
        return ms.value

    def opt_create(self, crit=REF_MEAN_RATIO, grid_scale=0.5, n_iter=30):
        st = refvs_lib().refvs_opt_create(self.h, int(crit), float(grid_scale), int(n_iter))
        if st != 0:
            raise RuntimeError(f"reference optimiser creation failed ({st})")

    def iterate(self, n=1):
        st = refvs_lib().refvs_opt_iterate(self.h, int(n))
        if st != 0:
            raise RuntimeError(f"reference iteration failed ({st})")

    def quality(self):
        return refvs_lib().refvs_opt_quality(self.h)

    def surface_state(self):
        """(initial positions [nSurf, 3], local surfaces [nSurf, 16] in the reference's layout
        p0, e0, e1, e2, a, b, c, numPoints (an int's bits), nearest initial vertex [nSurf])."""
        nS = self.info["nSurf"]
        x0 = np.zeros((nS, 3), np.float32)
        ls = np.zeros((nS, 16), np.float32)
        nn = np.zeros(nS, np.int32)
        st = refvs_lib().refvs_opt_surface_state(self.h, _p(x0), _p(ls), _p(nn))
        if st != 0:
            raise RuntimeError(f"reference surface state failed ({st})")
        return x0, ls, nn

    def surface_colour(self, cid):
        st = refvs_lib().refvs_opt_surface_colour(self.h, int(cid))
        if st != 0:
            raise RuntimeError(f"reference surface colour launch failed ({st})")

    def element_qualities(self):
        q = np.zeros(self.info["nE"], dtype=np.float32)
        st = refvs_lib().refvs_opt_element_qualities(self.h, _p(q))
        if st != 0:
            raise RuntimeError(f"reference element qualities failed ({st})")
        return q
