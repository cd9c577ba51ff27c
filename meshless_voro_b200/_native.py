"""ctypes binding of the C ABI in ``include/mvgpu.h`` (libmvgpu.so).

The library is loaded from ``meshless_voro_b200/_lib/``.  There is no CPU fallback:
if the CUDA library is missing or no device is usable, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# MVGPU_LIBRARY selects another build of the library (e.g. a tuning variant)
LIB_PATH = os.environ.get("MVGPU_LIBRARY") or os.path.join(_HERE, "_lib", "libmvgpu.so")

MV_OK = 0
MV_ERR_ARG = 1
MV_ERR_DEGENERATE = 2
MV_ERR_RING = 3
MV_ERR_DET = 4
MV_ERR_CAPACITY = 5
MV_ERR_CUDA = 6
MV_ERR_NO_DEVICE = 7
MV_ERR_OOM = 8

MV_PRECISION_FP64 = 0
MV_PRECISION_FILTERED = 1
MV_FACES_OWNED = 0
MV_FACES_ALL = 1

MV_CELLS_TETS = 1
MV_CELLS_WITH_FACES = 2

MV_PIPELINE_AUTO = 0
MV_PIPELINE_STAGED = 1
MV_PIPELINE_FUSED = 2

NO_SHIFT = 13

# every symbol include/mvgpu.h declares
EXPORTED = (
    "mv_options_default", "mv_strerror", "mv_version", "mv_context_create",
    "mv_context_destroy", "mv_context_last_stats", "mv_context_build_device",
    "mv_context_build", "mv_voronoi_build", "mv_voronoi_build_partial", "mv_voronoi_free",
    "mv_shift_from_code", "mv_voronoi_build_noalloc", "mv_context_build_cells_device",
    "mv_context_build_cells", "mv_context_build_batch_device", "mv_context_build_batch",
    "mv_tuning_set", "mv_tuning_lookup", "mv_tuning_count",
)


class Options(C.Structure):
    _fields_ = [("precision", C.c_int), ("face_mode", C.c_int),
                ("points_per_grid_cell", C.c_double), ("initial_radius", C.c_double),
                ("stream", C.c_void_p), ("pipeline", C.c_int), ("chunk_cells", C.c_int)]


class BuildStats(C.Structure):
    _fields_ = [(name, C.c_int64) for name in (
        "cells_built", "neighbours_clipped", "planes_added", "f32_undecided", "exact_tests",
        "extra_shells", "overflow_cells", "serial_rings", "staged_retries", "device_bytes",
        "kernel_launches")] + [
        (name, C.c_double) for name in ("ms_grid", "ms_cells", "ms_finalize", "ms_shell",
                                         "ms_clip", "ms_integrate", "ms_retry")] + [
        ("staged_wide", C.c_int64)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class DeviceVoronoi(C.Structure):
    _fields_ = [("n_cells", C.c_int64), ("n_faces", C.c_int64), ("n_connections", C.c_int64),
                ("cell_volume", C.c_void_p), ("cell_centroid", C.c_void_p),
                ("cell_safety_radius", C.c_void_p), ("cell_face_offset", C.c_void_p),
                ("cell_face_count", C.c_void_p), ("face_left", C.c_void_p),
                ("face_right", C.c_void_p), ("face_area", C.c_void_p),
                ("face_centroid", C.c_void_p), ("face_normal", C.c_void_p),
                ("face_shift_code", C.c_void_p), ("cell_face_connections", C.c_void_p),
                ("error_cell", C.c_int64)]


class HostVoronoi(C.Structure):
    _fields_ = [("n_cells", C.c_int64), ("n_faces", C.c_int64), ("n_connections", C.c_int64),
                ("dimensionality", C.c_int), ("periodic", C.c_int),
                ("anchor", C.c_double * 3), ("width", C.c_double * 3),
                ("cell_volume", C.POINTER(C.c_double)),
                ("cell_centroid", C.POINTER(C.c_double)),
                ("cell_safety_radius", C.POINTER(C.c_double)),
                ("cell_face_offset", C.POINTER(C.c_int64)),
                ("cell_face_count", C.POINTER(C.c_int32)),
                ("face_left", C.POINTER(C.c_int32)), ("face_right", C.POINTER(C.c_int32)),
                ("face_area", C.POINTER(C.c_double)),
                ("face_centroid", C.POINTER(C.c_double)),
                ("face_normal", C.POINTER(C.c_double)),
                ("face_shift_code", C.POINTER(C.c_uint8)),
                ("cell_face_connections", C.POINTER(C.c_int32)),
                ("error_cell", C.c_int64), ("_owner", C.c_void_p)]


class Cells(C.Structure):
    _fields_ = [(name, C.c_int64) for name in (
        "n_cells", "n_planes", "n_vertices", "n_tets", "n_faces", "n_face_vertices")] + [
        ("cell_plane_offset", C.c_void_p), ("plane_normal", C.c_void_p),
        ("plane_point", C.c_void_p), ("plane_right", C.c_void_p),
        ("plane_shift_code", C.c_void_p), ("cell_vertex_offset", C.c_void_p),
        ("vertex_loc", C.c_void_p), ("vertex_dual", C.c_void_p),
        ("cell_tet_offset", C.c_void_p), ("tet_vertices", C.c_void_p),
        ("tet_plane", C.c_void_p), ("cell_face_offset", C.c_void_p),
        ("face_plane", C.c_void_p), ("face_vertex_offset", C.c_void_p),
        ("face_vertices", C.c_void_p)]


class Job(C.Structure):
    """mv_job: one tessellation of a batch (its rows of the concatenated inputs)."""
    _fields_ = [("n", C.c_int64), ("anchor", C.c_double * 3), ("width", C.c_double * 3),
                ("dimensionality", C.c_int32), ("periodic", C.c_int32), ("has_mask", C.c_int32),
                ("reserved", C.c_int32)]


class TuningEntry(C.Structure):
    """mv_tuning_entry: the launch parameters of one dimensionality and size band."""
    _fields_ = [("dimensionality", C.c_int32), ("pipeline", C.c_int32), ("n_min", C.c_int64),
                ("n_max", C.c_int64), ("initial_radius", C.c_double),
                ("points_per_grid_cell", C.c_double), ("chunk_cells", C.c_int32),
                ("reserved", C.c_int32)]


class BatchVoronoi(C.Structure):
    _fields_ = [(name, C.c_int64) for name in ("n_jobs", "n_cells", "n_faces", "n_connections")] + [
        (name, C.POINTER(C.c_int64)) for name in (
            "job_cell_offset", "job_face_offset", "job_connection_offset")] + [
        (name, C.c_void_p) for name in (
            "cell_volume", "cell_centroid", "cell_safety_radius", "cell_face_offset",
            "cell_face_count", "face_left", "face_right", "face_area", "face_centroid",
            "face_normal", "face_shift_code", "cell_face_connections")] + [
        ("error_job", C.c_int64), ("error_cell", C.c_int64)]


_lib = None


def lib():
    """Load libmvgpu.so (raises if the CUDA library has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"CUDA library {LIB_PATH} is missing; build it with "
                "`python -m meshless_voro_b200.build` (nvcc, sm_100a)")
        L = C.CDLL(LIB_PATH)
        dp = C.POINTER(C.c_double)
        L.mv_options_default.argtypes = [C.POINTER(Options)]
        L.mv_options_default.restype = None
        L.mv_strerror.argtypes = [C.c_int]
        L.mv_strerror.restype = C.c_char_p
        L.mv_version.argtypes = []
        L.mv_version.restype = C.c_char_p
        L.mv_context_create.argtypes = [C.c_int, C.POINTER(C.c_void_p)]
        L.mv_context_create.restype = C.c_int
        L.mv_context_destroy.argtypes = [C.c_void_p]
        L.mv_context_destroy.restype = None
        L.mv_context_last_stats.argtypes = [C.c_void_p, C.POINTER(BuildStats)]
        L.mv_context_last_stats.restype = C.c_int
        L.mv_context_build_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, dp, dp,
                                              C.c_int, C.c_int, C.POINTER(Options),
                                              C.POINTER(DeviceVoronoi)]
        L.mv_context_build_device.restype = C.c_int
        L.mv_context_build.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, dp, dp,
                                       C.c_int, C.c_int, C.POINTER(Options),
                                       C.POINTER(C.POINTER(HostVoronoi))]
        L.mv_context_build.restype = C.c_int
        L.mv_voronoi_build.argtypes = [C.c_void_p, C.c_int64, dp, dp, C.c_int, C.c_int,
                                       C.POINTER(Options), C.POINTER(C.POINTER(HostVoronoi))]
        L.mv_voronoi_build.restype = C.c_int
        L.mv_voronoi_build_partial.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, dp, dp, C.c_int,
                                               C.c_int, C.POINTER(Options),
                                               C.POINTER(C.POINTER(HostVoronoi))]
        L.mv_voronoi_build_partial.restype = C.c_int
        L.mv_voronoi_free.argtypes = [C.POINTER(HostVoronoi)]
        L.mv_voronoi_free.restype = None
        L.mv_shift_from_code.argtypes = [C.c_int, dp, dp]
        L.mv_shift_from_code.restype = None
        L.mv_voronoi_build_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, dp, dp, C.c_int,
                                               C.c_int, C.POINTER(Options),
                                               C.POINTER(DeviceVoronoi), C.c_int64, C.c_int64]
        L.mv_voronoi_build_noalloc.restype = C.c_int
        L.mv_context_build_cells_device.argtypes = [
            C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, dp, dp, C.c_int, C.c_int,
            C.POINTER(Options), C.c_int, C.POINTER(DeviceVoronoi), C.POINTER(Cells)]
        L.mv_context_build_cells_device.restype = C.c_int
        L.mv_context_build_cells.argtypes = [
            C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, dp, dp, C.c_int, C.c_int,
            C.POINTER(Options), C.c_int, C.POINTER(C.POINTER(HostVoronoi)),
            C.POINTER(C.POINTER(Cells))]
        L.mv_context_build_cells.restype = C.c_int
        L.mv_context_build_batch_device.argtypes = [
            C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(Job), C.c_int64, C.POINTER(Options),
            C.POINTER(BatchVoronoi)]
        L.mv_context_build_batch_device.restype = C.c_int
        L.mv_context_build_batch.argtypes = [
            C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(Job), C.c_int64, C.POINTER(Options),
            C.POINTER(BatchVoronoi)]
        L.mv_context_build_batch.restype = C.c_int
        L.mv_tuning_set.argtypes = [C.POINTER(TuningEntry), C.c_int]
        L.mv_tuning_set.restype = C.c_int
        L.mv_tuning_lookup.argtypes = [C.c_int, C.c_int64, C.POINTER(TuningEntry)]
        L.mv_tuning_lookup.restype = C.c_int
        L.mv_tuning_count.argtypes = []
        L.mv_tuning_count.restype = C.c_int
        _lib = L
    return _lib


class MvError(RuntimeError):
    """A status code returned by the library (the reference panics in these cases)."""

    def __init__(self, status: int, error_cell: int = -1):
        self.status = status
        self.error_cell = error_cell
        msg = lib().mv_strerror(status).decode()
        if error_cell >= 0:
            msg += f" (cell {error_cell})"
        super().__init__(msg)


def check(status: int, error_cell: int = -1):
    if status != MV_OK:
        raise MvError(status, error_cell)
