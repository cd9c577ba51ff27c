"""ctypes wrapper over the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use
this module, and only as the checker / timed CPU restatement of the reference
algorithm (meshless_voronoi 0.7.2).  The product library never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

from . import build_oracle

_lib = None

FACES_ALL = 1
WITH_FACES = 2
BRUTE_FORCE = 4
EXPORT_CELLS = 8
EXPORT_TETS = 32
EXPORT_FACES = 64
NO_CSR = 16

STAT_FIELDS = ("n_nn", "n_planes", "n_vert", "max_vert", "n_exact", "n_shells", "n_cand", "pad")


def lib():
    global _lib
    if _lib is None:
        path = build_oracle.build()
        L = C.CDLL(path)
        P = C.c_void_p
        dp = C.POINTER(C.c_double)
        lp = C.POINTER(C.c_int64)
        ip = C.POINTER(C.c_int32)
        L.orc_build.restype = P
        L.orc_build.argtypes = [dp, C.c_int64, C.c_void_p, dp, dp, C.c_int, C.c_int, C.c_int,
                                C.c_int, C.c_double, C.c_double]
        for name in ("orc_status",):
            getattr(L, name).restype = C.c_int
            getattr(L, name).argtypes = [P]
        for name in ("orc_error_cell", "orc_n_faces", "orc_n_conn", "orc_n_planes_total",
                     "orc_n_verts_total"):
            getattr(L, name).restype = C.c_int64
            getattr(L, name).argtypes = [P]
        L.orc_copy_cells.argtypes = [P, dp, dp, dp, dp, lp, lp, lp]
        L.orc_copy_faces.argtypes = [P, lp, lp, dp, dp, dp, ip]
        L.orc_copy_conn.argtypes = [P, lp]
        L.orc_copy_stats.argtypes = [P, ip]
        L.orc_times.argtypes = [P, dp]
        L.orc_copy_cells_export.argtypes = [P, lp, dp, dp, lp, ip, lp, dp, ip]
        for name in ("orc_n_tets_total", "orc_n_cell_faces_total", "orc_n_face_vertices_total"):
            getattr(L, name).restype = C.c_int64
            getattr(L, name).argtypes = [P]
        L.orc_copy_tets.argtypes = [P, lp, dp, ip]
        L.orc_copy_face_lists.argtypes = [P, lp, ip, lp, ip]
        L.orc_free.argtypes = [P]
        L.orc_signed_volume_tet.restype = C.c_double
        L.orc_signed_volume_tet.argtypes = [dp] * 4
        L.orc_signed_area_tri.restype = C.c_double
        L.orc_signed_area_tri.argtypes = [dp] * 4
        L.orc_intersect_planes.restype = C.c_int
        L.orc_intersect_planes.argtypes = [dp] * 7
        L.orc_in_sphere_f64.restype = C.c_double
        L.orc_in_sphere_f64.argtypes = [dp] * 5
        L.orc_in_sphere_exact.restype = C.c_double
        L.orc_in_sphere_exact.argtypes = [lp] * 5
        L.orc_iloc.argtypes = [dp, dp, C.c_int, C.c_int, dp, lp]
        L.orc_half_space_clip.restype = C.c_double
        L.orc_half_space_clip.argtypes = [dp] * 3
        L.orc_simple_cycle.restype = C.c_int
        L.orc_simple_cycle.argtypes = [ip, C.c_int, C.c_int, ip, C.POINTER(C.c_int)]
        L.orc_clip_count.restype = C.c_int
        L.orc_clip_count.argtypes = [dp] * 4
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _lp(a):
    return a.ctypes.data_as(C.POINTER(C.c_int64))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _vec(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(3))


@dataclass
class OracleVoronoi:
    """Flat, reference-ordered output of one oracle build."""
    status: int
    error_cell: int
    volume: np.ndarray = None
    centroid: np.ndarray = None
    loc: np.ndarray = None
    safety_radius: np.ndarray = None
    face_offset: np.ndarray = None      # cell -> offset into cell_face_connections
    face_count: np.ndarray = None
    cell_face_begin: np.ndarray = None  # cell -> first face it emitted (n + 1 entries)
    face_left: np.ndarray = None
    face_right: np.ndarray = None       # -1 == boundary face
    face_area: np.ndarray = None
    face_centroid: np.ndarray = None
    face_normal: np.ndarray = None
    face_shift_code: np.ndarray = None  # 13 == no periodic shift
    cell_face_connections: np.ndarray = None
    stats: np.ndarray = None
    cells_export: dict = field(default=None)
    # wall seconds: setup (generators, boundary, grid), the per-cell loop, finalize
    times: tuple = (0.0, 0.0, 0.0)


def build(generators, anchor, width, dim=3, periodic=False, mask=None, nthreads=0, flags=0,
          ppc=0.0, r0_factor=0.0) -> OracleVoronoi:
    L = lib()
    g = np.ascontiguousarray(np.asarray(generators, dtype=np.float64).reshape(-1, 3))
    n = g.shape[0]
    m = None
    mp = None
    if mask is not None:
        m = np.ascontiguousarray(np.asarray(mask, dtype=np.uint8).reshape(n))
        mp = m.ctypes.data_as(C.c_void_p)
    a, w = _vec(anchor), _vec(width)
    h = L.orc_build(_dp(g), n, mp, _dp(a), _dp(w), int(dim), int(bool(periodic)), int(nthreads),
                    int(flags), float(ppc), float(r0_factor))
    try:
        st = L.orc_status(h)
        out = OracleVoronoi(status=st, error_cell=L.orc_error_cell(h))
        stats = np.zeros((n, len(STAT_FIELDS)), dtype=np.int32)
        L.orc_copy_stats(h, _ip(stats))
        out.stats = stats
        tt = np.zeros(3)
        L.orc_times(h, _dp(tt))
        out.times = tuple(float(x) for x in tt)
        if st != 0:
            return out
        F = L.orc_n_faces(h)
        Cn = L.orc_n_conn(h)
        out.volume = np.zeros(n)
        out.centroid = np.zeros((n, 3))
        out.loc = np.zeros((n, 3))
        out.safety_radius = np.zeros(n)
        out.face_offset = np.zeros(n, dtype=np.int64)
        out.face_count = np.zeros(n, dtype=np.int64)
        out.cell_face_begin = np.zeros(n + 1, dtype=np.int64)
        L.orc_copy_cells(h, _dp(out.volume), _dp(out.centroid), _dp(out.loc),
                         _dp(out.safety_radius), _lp(out.face_offset), _lp(out.face_count),
                         _lp(out.cell_face_begin))
        out.face_left = np.zeros(F, dtype=np.int64)
        out.face_right = np.zeros(F, dtype=np.int64)
        out.face_area = np.zeros(F)
        out.face_centroid = np.zeros((F, 3))
        out.face_normal = np.zeros((F, 3))
        out.face_shift_code = np.zeros(F, dtype=np.int32)
        L.orc_copy_faces(h, _lp(out.face_left), _lp(out.face_right), _dp(out.face_area),
                         _dp(out.face_centroid), _dp(out.face_normal), _ip(out.face_shift_code))
        out.cell_face_connections = np.zeros(Cn, dtype=np.int64)
        L.orc_copy_conn(h, _lp(out.cell_face_connections))
        if flags & EXPORT_CELLS:
            NP = L.orc_n_planes_total(h)
            NV = L.orc_n_verts_total(h)
            ex = dict(pl_off=np.zeros(n + 1, dtype=np.int64), pl_n=np.zeros((NP, 3)),
                      pl_p=np.zeros((NP, 3)), pl_right=np.zeros(NP, dtype=np.int64),
                      pl_code=np.zeros(NP, dtype=np.int32),
                      vx_off=np.zeros(n + 1, dtype=np.int64), vx_loc=np.zeros((NV, 3)),
                      vx_dual=np.zeros((NV, 3), dtype=np.int32))
            L.orc_copy_cells_export(h, _lp(ex["pl_off"]), _dp(ex["pl_n"]), _dp(ex["pl_p"]),
                                    _lp(ex["pl_right"]), _ip(ex["pl_code"]), _lp(ex["vx_off"]),
                                    _dp(ex["vx_loc"]), _ip(ex["vx_dual"]))
            out.cells_export = ex
        if flags & (EXPORT_TETS | EXPORT_FACES):
            ex = out.cells_export if out.cells_export is not None else {}
            if flags & EXPORT_TETS:
                T = L.orc_n_tets_total(h)
                ex["tet_off"] = np.zeros(n + 1, dtype=np.int64)
                ex["tet_v"] = np.zeros((T, 3, 3))
                ex["tet_plane"] = np.zeros(T, dtype=np.int32)
                L.orc_copy_tets(h, _lp(ex["tet_off"]), _dp(ex["tet_v"]), _ip(ex["tet_plane"]))
            if flags & EXPORT_FACES:
                Fc = L.orc_n_cell_faces_total(h)
                FV = L.orc_n_face_vertices_total(h)
                ex["cf_off"] = np.zeros(n + 1, dtype=np.int64)
                ex["cf_plane"] = np.zeros(Fc, dtype=np.int32)
                ex["fv_off"] = np.zeros(Fc + 1, dtype=np.int64)
                ex["fv"] = np.zeros(FV, dtype=np.int32)
                L.orc_copy_face_lists(h, _lp(ex["cf_off"]), _ip(ex["cf_plane"]), _lp(ex["fv_off"]),
                                      _ip(ex["fv"]))
            out.cells_export = ex
        return out
    finally:
        L.orc_free(h)


# ---- unit-level geometry entry points (reference geometry.rs / half_space.rs tests) ----
def signed_volume_tet(v0, v1, v2, v3):
    return lib().orc_signed_volume_tet(*[_dp(_vec(v)) for v in (v0, v1, v2, v3)])


def signed_area_tri(v0, v1, v2, t):
    return lib().orc_signed_area_tri(*[_dp(_vec(v)) for v in (v0, v1, v2, t)])


def intersect_planes(n0, p0, n1, p1, n2, p2):
    out = np.zeros(3)
    args = [_vec(v) for v in (n0, p0, n1, p1, n2, p2)]
    rc = lib().orc_intersect_planes(*[_dp(v) for v in args], _dp(out))
    if rc:
        raise ValueError("Degenerate 3-plane intersection!")
    return out


def in_sphere_f64(a, b, c, d, v):
    return lib().orc_in_sphere_f64(*[_dp(_vec(x)) for x in (a, b, c, d, v)])


def in_sphere_exact(a, b, c, d, v):
    arrs = [np.ascontiguousarray(np.asarray(x, dtype=np.int64).reshape(3)) for x in (a, b, c, d, v)]
    return lib().orc_in_sphere_exact(*[_lp(x) for x in arrs])


def iloc(anchor, width, loc, dim=3, periodic=False):
    out = np.zeros(3, dtype=np.int64)
    lib().orc_iloc(_dp(_vec(anchor)), _dp(_vec(width)), int(dim), int(periodic), _dp(_vec(loc)),
                   _lp(out))
    return out


def half_space_clip(n, p, v):
    return lib().orc_half_space_clip(_dp(_vec(n)), _dp(_vec(p)), _dp(_vec(v)))


def simple_cycle(tris, capacity):
    t = np.ascontiguousarray(np.asarray(tris, dtype=np.int32).reshape(-1, 3))
    out = np.zeros(max(capacity, 1), dtype=np.int32)
    ln = C.c_int(0)
    rc = lib().orc_simple_cycle(_ip(t), t.shape[0], int(capacity), _ip(out), C.byref(ln))
    if rc:
        raise ValueError("No suitable vertex found to extend boundary!")
    return out[: ln.value].tolist()


def clip_count(anchor, width, loc, ngb):
    return lib().orc_clip_count(*[_dp(_vec(v)) for v in (anchor, width, loc, ngb)])
