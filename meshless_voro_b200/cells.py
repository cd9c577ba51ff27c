"""The built convex cells and custom integrals (VoronoiIntegrator's cell view).

Mirrors the parts of meshless_voronoi 0.7.2 that hand out the cells themselves:
``ConvexCell`` (convex_cell.rs:249-262) with its ``HalfSpace`` planes
(half_space.rs:9-19) and ``Vertex`` list (convex_cell.rs:16-25), ``with_faces``
(convex_cell.rs:461-543) and the custom-integral protocol of integrals.rs
(``CellIntegral`` / ``FaceIntegral`` with ``init`` / ``collect`` / ``finalize``).

The cells, their decomposition into oriented tets and the sorted face-vertex lists are
built on the GPU (``mv_context_build_cells``); a custom integral is the user's own
code, fed the GPU's tets in the reference's order (``compute_cell_integral``,
convex_cell.rs:583-600), exactly as the crate feeds its tets to user integrals.  For
large builds, ``CellsArrays`` (tet_vertices, tet_plane and their per-cell offsets)
exposes the whole decomposition as arrays for vectorised integrals.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _native as N


@dataclass
class CellsArrays:
    """CSR arrays of the built cells, indexed by generator (empty for inactive cells)."""
    n_cells: int
    plane_offset: np.ndarray        # [n + 1]
    plane_normal: np.ndarray        # [P, 3]
    plane_point: np.ndarray         # [P, 3]
    plane_right: np.ndarray         # [P], -1: boundary
    plane_shift_code: np.ndarray    # [P]
    vertex_offset: np.ndarray       # [n + 1]
    vertex_loc: np.ndarray          # [V, 3]
    vertex_dual: np.ndarray         # [V, 3]
    tet_offset: Optional[np.ndarray] = None      # [n + 1]
    tet_vertices: Optional[np.ndarray] = None    # [T, 3, 3]
    tet_plane: Optional[np.ndarray] = None       # [T]
    face_offset: Optional[np.ndarray] = None     # [n + 1]
    face_plane: Optional[np.ndarray] = None      # [Fc]
    face_vertex_offset: Optional[np.ndarray] = None  # [Fc + 1]
    face_vertices: Optional[np.ndarray] = None   # [sum]

    @staticmethod
    def from_host(h: N.Cells) -> "CellsArrays":
        n = int(h.n_cells)
        P, V, T, Fc, FV = (int(h.n_planes), int(h.n_vertices), int(h.n_tets), int(h.n_faces),
                           int(h.n_face_vertices))

        def arr(ptr, count, ctype, shape):
            if not ptr:
                return None
            if count == 0:
                return np.zeros(shape, dtype=ctype)
            p = C.cast(ptr, C.POINTER(np.ctypeslib.as_ctypes_type(ctype)))
            return np.ctypeslib.as_array(p, shape=(count,)).copy().reshape(shape)

        out = CellsArrays(
            n_cells=n,
            plane_offset=arr(h.cell_plane_offset, n + 1, np.int64, (n + 1,)),
            plane_normal=arr(h.plane_normal, 3 * P, np.float64, (P, 3)),
            plane_point=arr(h.plane_point, 3 * P, np.float64, (P, 3)),
            plane_right=arr(h.plane_right, P, np.int32, (P,)),
            plane_shift_code=arr(h.plane_shift_code, P, np.uint8, (P,)),
            vertex_offset=arr(h.cell_vertex_offset, n + 1, np.int64, (n + 1,)),
            vertex_loc=arr(h.vertex_loc, 3 * V, np.float64, (V, 3)),
            vertex_dual=arr(h.vertex_dual, 3 * V, np.int32, (V, 3)))
        if h.tet_vertices:
            out.tet_offset = arr(h.cell_tet_offset, n + 1, np.int64, (n + 1,))
            out.tet_vertices = arr(h.tet_vertices, 9 * T, np.float64, (T, 3, 3))
            out.tet_plane = arr(h.tet_plane, T, np.int32, (T,))
        if h.face_vertices:
            out.face_offset = arr(h.cell_face_offset, n + 1, np.int64, (n + 1,))
            out.face_plane = arr(h.face_plane, Fc, np.int32, (Fc,))
            out.face_vertex_offset = arr(h.face_vertex_offset, Fc + 1, np.int64, (Fc + 1,))
            out.face_vertices = arr(h.face_vertices, FV, np.int32, (FV,))
        return out


class HalfSpace:
    """half_space.rs:9-19: a clipping plane (normal towards the cell) and its neighbour."""
    __slots__ = ("normal", "point", "right_idx", "shift")

    def __init__(self, normal, point, right_idx, shift):
        self.normal, self.point, self.right_idx, self.shift = normal, point, right_idx, shift


class Vertex:
    """convex_cell.rs:16-25: location and the three planes meeting there (ccw)."""
    __slots__ = ("loc", "dual")

    def __init__(self, loc, dual):
        self.loc, self.dual = loc, dual


class ConvexCell:
    """A built ConvexCell (convex_cell.rs:249-262); ``with_faces`` cells also carry the
    face lists of convex_cell.rs:667-731."""

    def __init__(self, a: CellsArrays, idx: int, loc, safety_radius: float, dimensionality: int,
                 width, with_faces: bool):
        from .voronoi import shift_from_code
        self._a, self.idx, self.loc = a, int(idx), np.asarray(loc, dtype=np.float64)
        self.safety_radius, self.dimensionality = safety_radius, dimensionality
        p0, p1 = int(a.plane_offset[idx]), int(a.plane_offset[idx + 1])
        self.clipping_planes = [
            HalfSpace(a.plane_normal[k], a.plane_point[k],
                      None if a.plane_right[k] < 0 else int(a.plane_right[k]),
                      shift_from_code(int(a.plane_shift_code[k]), width))
            for k in range(p0, p1)]
        v0, v1 = int(a.vertex_offset[idx]), int(a.vertex_offset[idx + 1])
        self.vertices = [Vertex(a.vertex_loc[k], tuple(int(d) for d in a.vertex_dual[k]))
                         for k in range(v0, v1)]
        self._with_faces = with_faces

    # ---- the decomposition (convex_cell.rs:203-235) ----
    def tets(self):
        """(v0, v1, v2, plane_idx) of the oriented tets, in the reference's order."""
        a = self._a
        if a.tet_vertices is None:
            raise RuntimeError("build the cells with MV_CELLS_TETS to decompose them")
        t0, t1 = int(a.tet_offset[self.idx]), int(a.tet_offset[self.idx + 1])
        return a.tet_vertices[t0:t1], a.tet_plane[t0:t1]

    def _plane_valid(self, k: int) -> bool:
        from .voronoi import Dimensionality
        return Dimensionality(self.dimensionality).vector_is_valid(self.clipping_planes[k].normal)

    def compute_cell_integral(self, integral, data=None):
        """convex_cell.rs:583-600"""
        it = _init_cell(integral, self, data)
        tv, _ = self.tets()
        for v in tv:
            it.collect(v[0], v[1], v[2], self.loc)
        return it.finalize()

    def compute_face_integrals(self, integral, data=None, mask=None, sym=False):
        """convex_cell.rs:604-664 (sym: skip faces shared with active cells of smaller index)."""
        from .voronoi import FaceIntegrator
        tv, tp = self.tets()
        its = {}
        for v, k in zip(tv, tp):
            k = int(k)
            if not self._plane_valid(k):
                continue
            if k not in its:
                h = self.clipping_planes[k]
                if (sym and h.shift is None and h.right_idx is not None and h.right_idx < self.idx
                        and mask[h.right_idx]):
                    continue
                its[k] = FaceIntegrator(self.idx, h.right_idx, h.shift,
                                        _init_face(integral, self, k, data))
            its[k]._integral.collect(v[0], v[1], v[2], self.loc)
        out = []
        for k in sorted(its):
            f = its[k]
            f._integral = f._integral.finalize()
            out.append(f)
        return out

    # ---- ConvexCell<WithFaces> (convex_cell.rs:667-731) ----
    def _faces(self):
        a = self._a
        if not self._with_faces or a.face_vertices is None:
            raise RuntimeError("faces are available after VoronoiIntegrator.with_faces()")
        return int(a.face_offset[self.idx]), int(a.face_offset[self.idx + 1])

    def face_count(self) -> int:
        f0, f1 = self._faces()
        return f1 - f0

    def _face_plane(self, face_idx: int) -> int:
        f0, _ = self._faces()
        return int(self._a.face_plane[f0 + face_idx])

    def clipping_plane(self, face_idx: int) -> HalfSpace:
        return self.clipping_planes[self._face_plane(face_idx)]

    def neighbour(self, face_idx: int):
        return self.clipping_plane(face_idx).right_idx

    def shift(self, face_idx: int):
        return self.clipping_plane(face_idx).shift

    def face_vertex_count(self, face_idx: int) -> int:
        return len(self.face_vertices(face_idx))

    def face_vertices(self, face_idx: int) -> np.ndarray:
        f0, _ = self._faces()
        a = self._a
        s, e = int(a.face_vertex_offset[f0 + face_idx]), int(a.face_vertex_offset[f0 + face_idx + 1])
        return a.face_vertices[s:e]


def _init_cell(integral, cell, data):
    if data is not None and hasattr(integral, "init_with_data"):
        return integral.init_with_data(cell, data)
    return integral.init(cell)


def _init_face(integral, cell, plane_idx, data):
    if data is not None and hasattr(integral, "init_with_data"):
        return integral.init_with_data(cell, plane_idx, data)
    return integral.init(cell, plane_idx)
