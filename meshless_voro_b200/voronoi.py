"""Host-side mirror of the meshless_voronoi 0.7.2 public API over the CUDA library.

Same names, argument meaning and error behaviour as the Rust crate:
``Voronoi.build`` (voronoi.rs:151-159), ``Voronoi.build_partial`` (voronoi.rs:181-190),
``VoronoiCell`` (voronoi_cell.rs:107-165), ``VoronoiFace`` (voronoi_face.rs:72-131),
``VoronoiIntegrator`` (voronoi.rs:527-828) with the built-in integrals of
integrals.rs.  Where the crate panics the library returns a status code and this
module raises ``MvError``.

Every build runs on the GPU through libmvgpu.so; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass
from typing import Iterator, Optional

import numpy as np

from . import _native as N


class Dimensionality(enum.IntEnum):
    """voronoi.rs:31-40"""
    OneD = 1
    TwoD = 2
    ThreeD = 3

    def vector_is_valid(self, v) -> bool:
        """voronoi.rs:42-49"""
        if self == Dimensionality.OneD:
            return v[1] == 0.0 and v[2] == 0.0
        if self == Dimensionality.TwoD:
            return v[2] == 0.0
        return True


PRECISION = {"fp64": N.MV_PRECISION_FP64, "filtered": N.MV_PRECISION_FILTERED}


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _vec3(v):
    return np.ascontiguousarray(np.asarray(v, dtype=np.float64).reshape(3))


def shift_from_code(code: int, width) -> Optional[np.ndarray]:
    """The reference's Option<DVec3> shift for a face shift code (rtree_nn.rs:27-33)."""
    if code == N.NO_SHIFT:
        return None
    out = np.zeros(3)
    N.lib().mv_shift_from_code(int(code), _dp(_vec3(width)), _dp(out))
    return out


PIPELINE = {"auto": N.MV_PIPELINE_AUTO, "staged": N.MV_PIPELINE_STAGED, "fused": N.MV_PIPELINE_FUSED}


def make_options(precision="filtered", face_mode=N.MV_FACES_OWNED, stream=None,
                 points_per_grid_cell=0.0, initial_radius=0.0, pipeline="auto",
                 chunk_cells=0) -> N.Options:
    o = N.Options()
    N.lib().mv_options_default(C.byref(o))
    o.precision = PRECISION[precision] if isinstance(precision, str) else int(precision)
    o.face_mode = int(face_mode)
    o.points_per_grid_cell = float(points_per_grid_cell)
    o.initial_radius = float(initial_radius)
    o.stream = stream
    o.pipeline = PIPELINE[pipeline] if isinstance(pipeline, str) else int(pipeline)
    o.chunk_cells = int(chunk_cells)
    return o


class Context:
    """A device, its CUDA stream and the reusable device workspace (mv_context)."""

    def __init__(self, device: int = -1):
        h = C.c_void_p()
        N.check(N.lib().mv_context_create(int(device), C.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            N.lib().mv_context_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def last_stats(self) -> dict:
        s = N.BuildStats()
        N.check(N.lib().mv_context_last_stats(self._h, C.byref(s)))
        return s.as_dict()

    def build_arrays(self, generators, mask, anchor, width, dimensionality, periodic,
                     precision="filtered", face_mode=N.MV_FACES_OWNED, **kw) -> "VoronoiArrays":
        """Host arrays in, host arrays out (mv_context_build); results are copied."""
        g = np.ascontiguousarray(np.asarray(generators, dtype=np.float64).reshape(-1, 3))
        n = g.shape[0]
        m = None
        if mask is not None:
            m = np.ascontiguousarray(np.asarray(mask, dtype=np.bool_).reshape(n)).view(np.uint8)
        a, w = _vec3(anchor), _vec3(width)
        opts = make_options(precision, face_mode, **kw)
        out = C.POINTER(N.HostVoronoi)()
        rc = N.lib().mv_context_build(self._h, g.ctypes.data_as(C.c_void_p),
                                      m.ctypes.data_as(C.c_void_p) if m is not None else None,
                                      n, _dp(a), _dp(w), int(dimensionality), int(bool(periodic)),
                                      C.byref(opts), C.byref(out))
        if rc != N.MV_OK:
            cell = out.contents.error_cell if out else -1
            raise N.MvError(rc, cell)
        return VoronoiArrays.from_host(out.contents, g, m, copy=True)

    def build_cells(self, generators, mask, anchor, width, dimensionality, periodic,
                    cells_flags=N.MV_CELLS_TETS, precision="filtered",
                    face_mode=N.MV_FACES_OWNED, **kw):
        """mv_context_build_cells: the Voronoi result and the built convex cells (host)."""
        from .cells import CellsArrays
        g = np.ascontiguousarray(np.asarray(generators, dtype=np.float64).reshape(-1, 3))
        n = g.shape[0]
        m = None
        if mask is not None:
            m = np.ascontiguousarray(np.asarray(mask, dtype=np.bool_).reshape(n)).view(np.uint8)
        a, w = _vec3(anchor), _vec3(width)
        opts = make_options(precision, face_mode, **kw)
        hv = C.POINTER(N.HostVoronoi)()
        hc = C.POINTER(N.Cells)()
        rc = N.lib().mv_context_build_cells(self._h, g.ctypes.data_as(C.c_void_p),
                                            m.ctypes.data_as(C.c_void_p) if m is not None else None,
                                            n, _dp(a), _dp(w), int(dimensionality),
                                            int(bool(periodic)), C.byref(opts), int(cells_flags),
                                            C.byref(hv), C.byref(hc))
        if rc != N.MV_OK:
            cell = hv.contents.error_cell if hv else -1
            raise N.MvError(rc, cell)
        return VoronoiArrays.from_host(hv.contents, g, m, copy=True), CellsArrays.from_host(hc.contents)

    def build_device(self, d_generators: int, d_mask: int, n: int, anchor, width,
                     dimensionality, periodic, precision="filtered",
                     face_mode=N.MV_FACES_OWNED, stream=None, **kw) -> N.DeviceVoronoi:
        """Device pointers in, device pointers (owned by this context) out."""
        a, w = _vec3(anchor), _vec3(width)
        opts = make_options(precision, face_mode, stream=stream, **kw)
        out = N.DeviceVoronoi()
        rc = N.lib().mv_context_build_device(self._h, C.c_void_p(d_generators),
                                             C.c_void_p(d_mask) if d_mask else None, int(n),
                                             _dp(a), _dp(w), int(dimensionality),
                                             int(bool(periodic)), C.byref(opts), C.byref(out))
        if rc != N.MV_OK:
            raise N.MvError(rc, out.error_cell)
        return out

    def build_batch(self, jobs, precision="filtered", face_mode=N.MV_FACES_OWNED, **kw) -> list:
        """mv_context_build_batch: many tessellations in one build (host in, host out).
        `jobs` holds dicts with generators, anchor, width, dimensionality, periodic and
        optionally mask; returns one VoronoiArrays per job, each what build_arrays
        returns for that job alone."""
        g, m, descs = batch_inputs(jobs)
        opts = make_options(precision, face_mode, **kw)
        out = N.BatchVoronoi()
        rc = N.lib().mv_context_build_batch(self._h, g.ctypes.data_as(C.c_void_p),
                                            m.ctypes.data_as(C.c_void_p) if m is not None else None,
                                            descs, len(jobs), C.byref(opts), C.byref(out))
        if rc != N.MV_OK:
            err = N.MvError(rc, out.error_cell)
            err.error_job = out.error_job
            raise err
        return batch_arrays(out, descs, g, m)

    def build_batch_device(self, d_generators: int, d_mask: int, descs, precision="filtered",
                           face_mode=N.MV_FACES_OWNED, stream=None, **kw) -> N.BatchVoronoi:
        """mv_context_build_batch_device: concatenated device inputs, device results."""
        opts = make_options(precision, face_mode, stream=stream, **kw)
        out = N.BatchVoronoi()
        rc = N.lib().mv_context_build_batch_device(self._h, C.c_void_p(d_generators),
                                                   C.c_void_p(d_mask) if d_mask else None, descs,
                                                   len(descs), C.byref(opts), C.byref(out))
        if rc != N.MV_OK:
            err = N.MvError(rc, out.error_cell)
            err.error_job = out.error_job
            raise err
        return out


class _DeviceArray:
    """A device pointer seen through __cuda_array_interface__ (no copy, not owned)."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr,
                                         "data": (int(ptr), False), "version": 3,
                                         "strides": None}


_DEVICE_FIELDS = (
    # name, element type, per-row width, row count ("n", "F" or "C")
    ("cell_volume", "<f8", 1, "n"), ("cell_centroid", "<f8", 3, "n"),
    ("cell_safety_radius", "<f8", 1, "n"), ("cell_face_offset", "<i8", 1, "n"),
    ("cell_face_count", "<i4", 1, "n"), ("face_left", "<i4", 1, "F"),
    ("face_right", "<i4", 1, "F"), ("face_area", "<f8", 1, "F"),
    ("face_centroid", "<f8", 3, "F"), ("face_normal", "<f8", 3, "F"),
    ("face_shift_code", "|u1", 1, "F"), ("cell_face_connections", "<i4", 1, "C"),
)


def device_tensors(dv, device=None) -> dict:
    """Zero-copy torch views of a device result (mv_device_voronoi, or a batch result's
    device arrays): one tensor per array, valid until the context's next build.  Arrays
    the build did not produce (the CSR of an MV_FACES_ALL build) are absent."""
    import torch
    rows = {"n": int(dv.n_cells), "F": int(dv.n_faces), "C": int(dv.n_connections)}
    dtypes = {"<f8": torch.float64, "<i8": torch.int64, "<i4": torch.int32, "|u1": torch.uint8}
    out = {}
    for name, typestr, width, dim in _DEVICE_FIELDS:
        ptr = getattr(dv, name)
        if not ptr:
            continue
        shape = (rows[dim], width) if width > 1 else (rows[dim],)
        if rows[dim] == 0:
            out[name] = torch.zeros(shape, dtype=dtypes[typestr], device=device or "cuda")
        else:
            out[name] = torch.as_tensor(_DeviceArray(ptr, shape, typestr), device=device)
    return out


def batch_inputs(jobs):
    """Concatenated generators, concatenated mask (or None) and the mv_job descriptors of a
    sequence of tessellations, each a dict with generators, anchor, width, dimensionality,
    periodic and optionally mask (the layout mv_context_build_batch reads)."""
    gens, masks, descs = [], [], (N.Job * len(jobs))()
    any_mask = any(j.get("mask") is not None for j in jobs)
    for k, j in enumerate(jobs):
        g = np.asarray(j["generators"], dtype=np.float64).reshape(-1, 3)
        gens.append(g)
        d = descs[k]
        d.n = g.shape[0]
        d.anchor[:] = list(_vec3(j["anchor"]))
        d.width[:] = list(_vec3(j["width"]))
        d.dimensionality = int(j["dimensionality"])
        d.periodic = int(bool(j["periodic"]))
        d.has_mask = int(j.get("mask") is not None)
        if any_mask:
            m = j.get("mask")
            masks.append(np.ones(g.shape[0], np.uint8) if m is None
                         else np.asarray(m, dtype=np.bool_).reshape(g.shape[0]).view(np.uint8))
    g = np.ascontiguousarray(np.concatenate(gens) if gens else np.zeros((0, 3)))
    m = np.ascontiguousarray(np.concatenate(masks)) if any_mask else None
    return g, m, descs


def batch_arrays(bv: N.BatchVoronoi, descs, generators: np.ndarray, mask_u8) -> list:
    """Splits a host batch result into one VoronoiArrays per tessellation (copies)."""
    nj = int(bv.n_jobs)
    n, F, Cn = int(bv.n_cells), int(bv.n_faces), int(bv.n_connections)

    def full(ptr, count, ctype, dtype, width=1):
        if count == 0 or not ptr:
            return np.zeros((0, width) if width > 1 else 0, dtype=dtype)
        a = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ctype)), shape=(count * width,))
        return a.reshape(count, width) if width > 1 else a

    has_csr = bool(bv.cell_face_offset)
    vol = full(bv.cell_volume, n, C.c_double, np.float64)
    cen = full(bv.cell_centroid, n, C.c_double, np.float64, 3)
    sr = full(bv.cell_safety_radius, n, C.c_double, np.float64)
    foff = full(bv.cell_face_offset, n, C.c_int64, np.int64) if has_csr else None
    fcnt = full(bv.cell_face_count, n, C.c_int32, np.int32) if has_csr else None
    fl = full(bv.face_left, F, C.c_int32, np.int32)
    fr = full(bv.face_right, F, C.c_int32, np.int32)
    fa = full(bv.face_area, F, C.c_double, np.float64)
    fc = full(bv.face_centroid, F, C.c_double, np.float64, 3)
    fn = full(bv.face_normal, F, C.c_double, np.float64, 3)
    fs = full(bv.face_shift_code, F, C.c_uint8, np.uint8)
    conn = full(bv.cell_face_connections, Cn, C.c_int32, np.int32) if has_csr else None
    co, fo, no = bv.job_cell_offset, bv.job_face_offset, bv.job_connection_offset
    res = []
    for j in range(nj):
        c0, c1, f0, f1 = co[j], co[j + 1], fo[j], fo[j + 1]
        d = descs[j]
        dim = int(d.dimensionality)
        loc = generators[c0:c1].copy()
        if dim == 1:
            loc[:, 1:] = 0.0
        elif dim == 2:
            loc[:, 2] = 0.0
        if d.has_mask and mask_u8 is not None:
            loc[mask_u8[c0:c1] == 0] = 0.0
        res.append(VoronoiArrays(
            n_cells=c1 - c0, anchor=np.array(d.anchor[:]), width=np.array(d.width[:]),
            dimensionality=dim, periodic=bool(d.periodic),
            cell_volume=vol[c0:c1].copy(), cell_centroid=cen[c0:c1].copy(), cell_loc=loc,
            cell_safety_radius=sr[c0:c1].copy(),
            cell_face_offset=foff[c0:c1].astype(np.int64) if has_csr else None,
            cell_face_count=fcnt[c0:c1].astype(np.int64) if has_csr else None,
            face_left=fl[f0:f1].astype(np.int64), face_right=fr[f0:f1].astype(np.int64),
            face_area=fa[f0:f1].copy(), face_centroid=fc[f0:f1].copy(),
            face_normal=fn[f0:f1].copy(), face_shift_code=fs[f0:f1].astype(np.int32),
            cell_face_connections=conn[no[j]:no[j + 1]].astype(np.int64) if has_csr else None))
    return res


_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(-1)
    return _default_ctx


@dataclass
class VoronoiArrays:
    """Flat, reference-ordered results of one build (numpy, host)."""
    n_cells: int
    anchor: np.ndarray
    width: np.ndarray
    dimensionality: int
    periodic: bool
    cell_volume: np.ndarray
    cell_centroid: np.ndarray
    cell_loc: np.ndarray
    cell_safety_radius: np.ndarray
    cell_face_offset: Optional[np.ndarray]
    cell_face_count: Optional[np.ndarray]
    face_left: np.ndarray
    face_right: np.ndarray
    face_area: np.ndarray
    face_centroid: np.ndarray
    face_normal: np.ndarray
    face_shift_code: np.ndarray
    cell_face_connections: Optional[np.ndarray]

    @staticmethod
    def from_host(hv: N.HostVoronoi, generators: np.ndarray, mask_u8, copy=True) -> "VoronoiArrays":
        n, F, Cn = int(hv.n_cells), int(hv.n_faces), int(hv.n_connections)

        def arr(ptr, count, dtype, shape=None):
            if count == 0 or not ptr:
                a = np.zeros(0 if shape is None else (0,) + shape[1:], dtype=dtype)
                return a
            a = np.ctypeslib.as_array(ptr, shape=(count,))
            a = a.astype(dtype, copy=True) if copy else a
            return a.reshape(shape) if shape else a

        dim = int(hv.dimensionality)
        loc = generators.copy()
        if dim == 1:
            loc[:, 1:] = 0.0
        elif dim == 2:
            loc[:, 2] = 0.0
        if mask_u8 is not None:
            loc[mask_u8 == 0] = 0.0
        has_csr = bool(hv.cell_face_offset)
        return VoronoiArrays(
            n_cells=n, anchor=np.array(hv.anchor[:]), width=np.array(hv.width[:]),
            dimensionality=dim, periodic=bool(hv.periodic),
            cell_volume=arr(hv.cell_volume, n, np.float64),
            cell_centroid=arr(hv.cell_centroid, 3 * n, np.float64, (n, 3)),
            cell_loc=loc,
            cell_safety_radius=arr(hv.cell_safety_radius, n, np.float64),
            cell_face_offset=arr(hv.cell_face_offset, n, np.int64) if has_csr else None,
            cell_face_count=arr(hv.cell_face_count, n, np.int64) if has_csr else None,
            face_left=arr(hv.face_left, F, np.int64),
            face_right=arr(hv.face_right, F, np.int64),
            face_area=arr(hv.face_area, F, np.float64),
            face_centroid=arr(hv.face_centroid, 3 * F, np.float64, (F, 3)),
            face_normal=arr(hv.face_normal, 3 * F, np.float64, (F, 3)),
            face_shift_code=arr(hv.face_shift_code, F, np.int32),
            cell_face_connections=arr(hv.cell_face_connections, Cn, np.int64) if has_csr else None,
        )


class VoronoiCell:
    """voronoi_cell.rs:11-165 (a view into a Voronoi)."""

    __slots__ = ("_v", "_i")

    def __init__(self, voronoi: "Voronoi", idx: int):
        self._v = voronoi
        self._i = idx

    def loc(self) -> np.ndarray:
        return self._v.arrays.cell_loc[self._i]

    def centroid(self) -> np.ndarray:
        return self._v.arrays.cell_centroid[self._i]

    def volume(self) -> float:
        return float(self._v.arrays.cell_volume[self._i])

    def safety_radius(self) -> float:
        return float(self._v.arrays.cell_safety_radius[self._i])

    def face_connections_offset(self) -> int:
        return int(self._v.arrays.cell_face_offset[self._i])

    def face_count(self) -> int:
        return int(self._v.arrays.cell_face_count[self._i])

    def face_indices(self, voronoi: "Voronoi" = None) -> np.ndarray:
        v = voronoi or self._v
        o = self.face_connections_offset()
        return v.arrays.cell_face_connections[o:o + self.face_count()]

    def faces(self, voronoi: "Voronoi" = None) -> Iterator["VoronoiFace"]:
        v = voronoi or self._v
        for f in self.face_indices(v):
            yield VoronoiFace(v, int(f))

    def neighbour_ids(self, voronoi: "Voronoi" = None) -> Iterator[int]:
        """voronoi_cell.rs:141-153: other side of every non-periodic, non-boundary face.
        An inactive cell has index 0 in the reference (VoronoiCell::default)."""
        v = voronoi or self._v
        a = v.arrays
        my_idx = self._i if a.cell_volume[self._i] != 0.0 or not v._partial else 0
        for f in self.face_indices(v):
            if a.face_shift_code[f] != N.NO_SHIFT or a.face_right[f] < 0:
                continue
            yield int(a.face_right[f]) if a.face_left[f] == my_idx else int(a.face_left[f])


class VoronoiFace:
    """voronoi_face.rs:48-132 (a view into a Voronoi)."""

    __slots__ = ("_v", "_f")

    def __init__(self, voronoi: "Voronoi", idx: int):
        self._v = voronoi
        self._f = idx

    def left(self) -> int:
        return int(self._v.arrays.face_left[self._f])

    def right(self) -> Optional[int]:
        r = int(self._v.arrays.face_right[self._f])
        return None if r < 0 else r

    def area(self) -> float:
        return float(self._v.arrays.face_area[self._f])

    def centroid(self) -> np.ndarray:
        return self._v.arrays.face_centroid[self._f]

    def normal(self) -> np.ndarray:
        return self._v.arrays.face_normal[self._f]

    def shift(self) -> Optional[np.ndarray]:
        return shift_from_code(int(self._v.arrays.face_shift_code[self._f]), self._v.width())

    def is_periodic(self) -> bool:
        return int(self._v.arrays.face_shift_code[self._f]) != N.NO_SHIFT

    def is_boundary(self) -> bool:
        return int(self._v.arrays.face_right[self._f]) < 0


class Voronoi:
    """voronoi.rs:110-408"""

    def __init__(self, arrays: VoronoiArrays, partial: bool = False):
        self.arrays = arrays
        self._partial = partial

    @staticmethod
    def build(generators, anchor, width, dimensionality=Dimensionality.ThreeD, periodic=False, *,
              precision="filtered", context: Context = None, **kw) -> "Voronoi":
        ctx = context or default_context()
        a = ctx.build_arrays(generators, None, anchor, width, int(dimensionality), periodic,
                             precision=precision, **kw)
        return Voronoi(a)

    @staticmethod
    def build_partial(generators, mask, anchor, width, dimensionality=Dimensionality.ThreeD,
                      periodic=False, *, precision="filtered", context: Context = None,
                      **kw) -> "Voronoi":
        ctx = context or default_context()
        a = ctx.build_arrays(generators, mask, anchor, width, int(dimensionality), periodic,
                             precision=precision, **kw)
        return Voronoi(a, partial=True)

    def anchor(self) -> np.ndarray:
        return self.arrays.anchor

    def width(self) -> np.ndarray:
        return self.arrays.width

    def cells(self):
        return [VoronoiCell(self, i) for i in range(self.arrays.n_cells)]

    def faces(self):
        return [VoronoiFace(self, f) for f in range(len(self.arrays.face_left))]

    def cell_face_connections(self) -> np.ndarray:
        return self.arrays.cell_face_connections

    def dimensionality(self) -> int:
        return self.arrays.dimensionality

    def hdf5_datasets(self) -> dict:
        """The datasets Voronoi::write_to_hdf5 writes (voronoi.rs:432-491), by HDF5 path:
        Cells/{Volume, FaceConnectionsOffset, FaceCount, Centroid, Generator},
        Faces/{Area, Centroid, Normal} (and Start, End for 2D) and CellFaceConnections,
        in its types (usize as uint64).  The 2D face end points are
        centroid -/+ 0.5 * area * (normal x Z) in glam's operation order
        (voronoi.rs:462-483), so they are the reference's binary64 values."""
        a = self.arrays
        if a.cell_face_connections is None:
            raise ValueError("the HDF5 layout needs the cell -> face connections (MV_FACES_OWNED)")
        d = {
            "Cells/Volume": np.asarray(a.cell_volume, dtype=np.float64),
            "Cells/FaceConnectionsOffset": np.asarray(a.cell_face_offset, dtype=np.uint64),
            "Cells/FaceCount": np.asarray(a.cell_face_count, dtype=np.uint64),
            "Cells/Centroid": np.asarray(a.cell_centroid, dtype=np.float64).reshape(-1, 3),
            "Cells/Generator": np.asarray(a.cell_loc, dtype=np.float64).reshape(-1, 3),
            "Faces/Area": np.asarray(a.face_area, dtype=np.float64),
            "Faces/Centroid": np.asarray(a.face_centroid, dtype=np.float64).reshape(-1, 3),
            "Faces/Normal": np.asarray(a.face_normal, dtype=np.float64).reshape(-1, 3),
        }
        if a.dimensionality == 2:
            n, c = d["Faces/Normal"], d["Faces/Centroid"]
            # DVec3::cross(n, Z): (n.y z - Z.y n.z, n.z Z.x - Z.z n.x, n.x Z.y - Z.x n.y)
            cross = np.stack([n[:, 1] * 1.0 - 0.0 * n[:, 2], n[:, 2] * 0.0 - 1.0 * n[:, 0],
                              n[:, 0] * 0.0 - 0.0 * n[:, 1]], axis=1)
            direction = d["Faces/Area"][:, None] * cross
            d["Faces/Start"] = c - 0.5 * direction
            d["Faces/End"] = c + 0.5 * direction
        d["CellFaceConnections"] = np.asarray(a.cell_face_connections, dtype=np.uint64)
        return d

    def write_to_hdf5(self, filename) -> None:
        """Voronoi::write_to_hdf5 (voronoi.rs:432-491): groups Cells and Faces and the
        top-level CellFaceConnections, through h5py (the crate needs its `hdf5` feature
        for this; here the h5py package)."""
        try:
            import h5py
        except ImportError as e:
            raise RuntimeError("write_to_hdf5 needs the h5py package, which is not installed; "
                               "save_datasets writes the same datasets to an .npz") from e
        with h5py.File(filename, "w") as f:
            for path, data in self.hdf5_datasets().items():
                f.create_dataset(path, data=data)

    def save_datasets(self, filename) -> None:
        """The datasets of write_to_hdf5 in an .npz archive, keyed by their HDF5 paths."""
        np.savez(filename, **self.hdf5_datasets())

    def periodic(self) -> bool:
        return self.arrays.periodic


# ------------------------------------------------------------ integrals.rs --
# The built-in integrals: the device computes them for every build; they also follow the
# crate's protocol (init / collect / finalize over oriented tets), restated with glam's
# operation order in binary64 (geometry.rs:82-100), for cells decomposed with faces.
def _sub(a, b):
    return (a[0] - b[0], a[1] - b[1], a[2] - b[2])


def _dot(a, b):
    return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]


def _cross(a, b):
    return (a[1] * b[2] - b[1] * a[2], a[2] * b[0] - b[2] * a[0], a[0] * b[1] - b[0] * a[1])


def signed_volume_tet(v0, v1, v2, v3) -> float:
    """geometry.rs:82-88: DMat3::from_cols(v1-v0, v2-v0, v3-v0).determinant() / 6"""
    c0, c1, c2 = _sub(v1, v0), _sub(v2, v0), _sub(v3, v0)
    return _dot(c2, _cross(c0, c1)) / 6.0


def signed_area_tri(v0, v1, v2, t) -> float:
    """geometry.rs:95-100"""
    c = _cross(_sub(v1, v0), _sub(v2, v0))
    n = (0.5 * c[0], 0.5 * c[1], 0.5 * c[2])
    sign = np.copysign(1.0, _dot(_sub(t, v0), n))
    return float(np.sqrt(_dot(n, n))) * float(sign)


def _f3(v):
    return (float(v[0]), float(v[1]), float(v[2]))


class VolumeIntegral:
    """integrals.rs:124-142"""
    __slots__ = ("volume",)

    def __init__(self, volume=0.0):
        self.volume = volume

    @classmethod
    def init(cls, cell):
        return cls(0.0)

    def collect(self, v0, v1, v2, gen):
        self.volume += signed_volume_tet(_f3(v0), _f3(v1), _f3(v2), _f3(gen))

    def finalize(self):
        return self


class VolumeCentroidIntegral:
    """integrals.rs:69-106"""
    __slots__ = ("volume", "centroid")

    def __init__(self, volume=0.0, centroid=None):
        self.volume = volume
        self.centroid = np.zeros(3) if centroid is None else centroid

    @classmethod
    def init(cls, cell):
        return cls(0.0, (0.0, 0.0, 0.0))

    def collect(self, v0, v1, v2, gen):
        a, b, c, g = _f3(v0), _f3(v1), _f3(v2), _f3(gen)
        vol = signed_volume_tet(a, b, c, g)
        self.volume += vol
        s = tuple(((a[i] + b[i]) + c[i]) + g[i] for i in range(3))
        self.centroid = tuple(self.centroid[i] + vol * s[i] for i in range(3))

    def finalize(self):
        norm = 0.25 / self.volume if self.volume > 0.0 else 0.0
        self.centroid = np.array([self.centroid[i] * norm for i in range(3)])
        return self


class AreaIntegral:
    """integrals.rs:343-361"""
    __slots__ = ("area",)

    def __init__(self, area=0.0, centroid=None):
        self.area = area

    @classmethod
    def init(cls, cell, clipping_plane_idx):
        return cls(0.0)

    def collect(self, v0, v1, v2, gen):
        self.area += signed_area_tri(_f3(v0), _f3(v1), _f3(v2), _f3(gen))

    def finalize(self):
        return self


class AreaCentroidIntegral:
    """integrals.rs:283-320"""
    __slots__ = ("area", "centroid")

    def __init__(self, area=0.0, centroid=None):
        self.area = area
        self.centroid = np.zeros(3) if centroid is None else centroid

    @classmethod
    def init(cls, cell, clipping_plane_idx):
        return cls(0.0, (0.0, 0.0, 0.0))

    def collect(self, v0, v1, v2, gen):
        a, b, c = _f3(v0), _f3(v1), _f3(v2)
        ar = signed_area_tri(a, b, c, _f3(gen))
        self.area += ar
        s = tuple((a[i] + b[i]) + c[i] for i in range(3))
        self.centroid = tuple(self.centroid[i] + ar * s[i] for i in range(3))

    def finalize(self):
        norm = 1.0 / (3.0 * self.area) if self.area > 0.0 else 0.0
        self.centroid = np.array([self.centroid[i] * norm for i in range(3)])
        return self


_BUILTIN_CELL = (VolumeIntegral, VolumeCentroidIntegral)
_BUILTIN_FACE = (AreaIntegral, AreaCentroidIntegral)


class FaceIntegrator:
    """integrals.rs:204-259"""
    __slots__ = ("_left", "_right", "_shift", "_integral")

    def __init__(self, left, right, shift, integral):
        self._left, self._right, self._shift, self._integral = left, right, shift, integral

    def left(self):
        return self._left

    def right(self):
        return self._right

    def shift(self):
        return self._shift

    def integral(self):
        return self._integral


class VoronoiIntegrator:
    """voronoi.rs:527-828: the built-in integrals come from the device build; custom
    integrals (any class with the crate's init / collect / finalize protocol) and the
    cells themselves come from a cells build (mv_context_build_cells), whose tets are
    the reference's decomposition computed on the GPU."""

    def __init__(self, generators, mask, anchor, width, dimensionality, periodic, precision,
                 context, with_faces=False):
        self._g = np.ascontiguousarray(np.asarray(generators, dtype=np.float64).reshape(-1, 3))
        self._mask = None if mask is None else np.asarray(mask, dtype=bool).reshape(-1)
        self._anchor, self._width = _vec3(anchor), _vec3(width)
        self._dim = int(dimensionality)
        self._periodic = bool(periodic)
        self._precision = precision
        self._ctx = context or default_context()
        self._with_faces = with_faces
        self._cache = {}

    @staticmethod
    def build(generators, mask, anchor, width, dimensionality=Dimensionality.ThreeD,
              periodic=False, *, precision="filtered", context: Context = None):
        return VoronoiIntegrator(generators, mask, anchor, width, dimensionality, periodic,
                                 precision, context)

    def with_faces(self) -> "VoronoiIntegrator":
        """voronoi.rs:621-638 / convex_cell.rs:461-466: 3D only (the crate panics)."""
        if self._dim != 3:
            raise ValueError("Can only convert to WithFaces in 3D!")
        return VoronoiIntegrator(self._g, self._mask, self._anchor, self._width, self._dim,
                                 self._periodic, self._precision, self._ctx, with_faces=True)

    def _run(self, face_mode) -> VoronoiArrays:
        if face_mode not in self._cache:
            self._cache[face_mode] = self._ctx.build_arrays(
                self._g, self._mask, self._anchor, self._width, self._dim, self._periodic,
                precision=self._precision, face_mode=face_mode)
        return self._cache[face_mode]

    def _cells(self):
        """(VoronoiArrays, CellsArrays) of a cells build (cached)."""
        if "cells" not in self._cache:
            flags = N.MV_CELLS_TETS | (N.MV_CELLS_WITH_FACES if self._with_faces else 0)
            self._cache["cells"] = self._ctx.build_cells(
                self._g, self._mask, self._anchor, self._width, self._dim, self._periodic,
                cells_flags=flags, precision=self._precision)
        return self._cache["cells"]

    def _active(self):
        n = self._g.shape[0]
        return np.ones(n, dtype=bool) if self._mask is None else self._mask

    def cells_arrays(self):
        """All built cells as CSR arrays (planes, vertices, tets, faces) for vectorised
        custom integrals."""
        return self._cells()[1]

    def get_cell_at(self, index: int):
        """voronoi.rs:647-649: the ConvexCell of a generator, None if it was not built."""
        from .cells import ConvexCell
        if not self._active()[index]:
            return None
        va, ca = self._cells()
        return ConvexCell(ca, index, va.cell_loc[index], float(va.cell_safety_radius[index]),
                          self._dim, self._width, self._with_faces)

    def cells_iter(self) -> Iterator:
        """voronoi.rs:655-657"""
        for i in np.nonzero(self._active())[0]:
            yield self.get_cell_at(int(i))

    def compute_cell_integrals(self, integral=VolumeCentroidIntegral):
        """voronoi.rs:668-673: one integral per active cell, in cell order."""
        if integral in _BUILTIN_CELL and not self._with_faces:
            a = self._run(N.MV_FACES_OWNED)
            idx = np.nonzero(self._active())[0]
            if integral is VolumeIntegral:
                return [VolumeIntegral(float(a.cell_volume[i])) for i in idx]
            return [VolumeCentroidIntegral(float(a.cell_volume[i]), a.cell_centroid[i]) for i in idx]
        return [c.compute_cell_integral(integral) for c in self.cells_iter()]

    def compute_cell_integrals_with_data(self, integral, extra_data):
        """voronoi.rs:679-698"""
        return [c.compute_cell_integral(integral, extra_data[c.idx]) for c in self.cells_iter()]

    def _faces(self, a: VoronoiArrays, integral):
        out = []
        for f in range(len(a.face_left)):
            r = int(a.face_right[f])
            shift = shift_from_code(int(a.face_shift_code[f]), a.width)
            if integral is AreaIntegral:
                val = AreaIntegral(float(a.face_area[f]))
            else:
                val = AreaCentroidIntegral(float(a.face_area[f]), a.face_centroid[f])
            out.append(FaceIntegrator(int(a.face_left[f]), None if r < 0 else r, shift, val))
        return out

    def _custom_faces(self, integral, sym, extra_data=None):
        mask = self._active()
        out = []
        for c in self.cells_iter():
            data = None if extra_data is None else extra_data[c.idx]
            out.extend(c.compute_face_integrals(integral, data, mask, sym))
        return out

    def compute_face_integrals(self, integral=AreaCentroidIntegral):
        """voronoi.rs:709-714: every face of every active cell (non-symmetric)."""
        if integral in _BUILTIN_FACE and not self._with_faces:
            return self._faces(self._run(N.MV_FACES_ALL), integral)
        return self._custom_faces(integral, sym=False)

    def compute_face_integrals_sym(self, integral=AreaCentroidIntegral):
        """voronoi.rs:725-732: each face once."""
        if integral in _BUILTIN_FACE and not self._with_faces:
            return self._faces(self._run(N.MV_FACES_OWNED), integral)
        return self._custom_faces(integral, sym=True)

    def compute_face_integrals_with_data(self, integral, extra_data):
        """voronoi.rs:749-769"""
        return self._custom_faces(integral, sym=False, extra_data=extra_data)

    def compute_face_integrals_sym_with_data(self, integral, extra_data):
        """voronoi.rs:784-808"""
        return self._custom_faces(integral, sym=True, extra_data=extra_data)

    def to_voronoi(self) -> Voronoi:
        """From<&VoronoiIntegrator> for Voronoi (voronoi.rs:494-513)."""
        return Voronoi(self._run(N.MV_FACES_OWNED), partial=self._mask is not None)
