"""meshless_voro_b200 -- B200-native (sm_100a) per-cell Voronoi construction.

Drop-in for the cell-construction path of the Rust crate meshless_voronoi 0.7.2:
the C ABI is ``include/mvgpu.h`` (libmvgpu.so); this package mirrors the crate's
public API on top of it.
"""
from ._native import MvError  # noqa: F401
from .voronoi import (  # noqa: F401
    AreaCentroidIntegral,
    AreaIntegral,
    Context,
    Dimensionality,
    FaceIntegrator,
    Voronoi,
    VoronoiArrays,
    VoronoiCell,
    VoronoiFace,
    VoronoiIntegrator,
    VolumeCentroidIntegral,
    VolumeIntegral,
    default_context,
    shift_from_code,
)

__all__ = [
    "AreaCentroidIntegral", "AreaIntegral", "Context", "Dimensionality", "FaceIntegrator",
    "MvError", "Voronoi", "VoronoiArrays", "VoronoiCell", "VoronoiFace", "VoronoiIntegrator",
    "VolumeCentroidIntegral", "VolumeIntegral", "default_context", "shift_from_code",
]
