"""Shared checks restating the reference's test helpers (voronoi.rs:363-408)."""
from __future__ import annotations

import math

import numpy as np


def approx_eq(a, b, epsilon=np.finfo(float).eps, ulps=4):
    """float_cmp::approx_eq!(f64, a, b, epsilon, ulps)"""
    if abs(a - b) <= epsilon:
        return True
    if (a < 0) != (b < 0):
        return a == b
    ia = np.float64(a).view(np.int64)
    ib = np.float64(b).view(np.int64)
    return abs(int(ia) - int(ib)) <= ulps


def vector_is_valid(dim, v):
    if dim == 1:
        return v[1] == 0.0 and v[2] == 0.0
    if dim == 2:
        return v[2] == 0.0
    return True


def consistency_check(r, dim, width):
    """Voronoi::consistency_check (voronoi.rs:363-408) on flat result arrays
    (volume, face_offset, face_count, face_area, face_normal, cell_face_connections)."""
    total = 0.0
    all_active = True
    n = len(r.volume) if hasattr(r, "volume") else len(r.cell_volume)
    vol = r.volume if hasattr(r, "volume") else r.cell_volume
    off = r.face_offset if hasattr(r, "face_offset") else r.cell_face_offset
    cnt = r.face_count if hasattr(r, "face_count") else r.cell_face_count
    for i in range(n):
        v = vol[i]
        if v == 0.0:
            all_active = False
            continue
        total += v
        fs = r.cell_face_connections[off[i]:off[i] + cnt[i]]
        area = 0.0
        for f in fs:
            assert vector_is_valid(dim, r.face_normal[f])
            area += r.face_area[f]
        if dim == 3:
            radius = (0.25 * 3.0 / math.pi * v) ** (1.0 / 3.0)
            assert area > 4.0 * math.pi * radius * radius, (i, area)
        elif dim == 2:
            radius = math.sqrt(v / math.pi)
            assert area > 2.0 * math.pi * radius, (i, area)
        else:
            assert approx_eq(area, 2.0), (i, area)
    if all_active and dim == 3:
        box = float(width[0] * width[1] * width[2])
        assert approx_eq(total, box, epsilon=box * 1e-11, ulps=4), (total, box)


REL_TOL = 1e-12  # integrals within 1e-12 relative of the oracle


def _rel_err(a, b, scale):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.size == 0:
        return 0.0
    return float(np.max(np.abs(a - b) / (np.abs(b) + scale)))


def compare(gpu, orc, faces_all=False):
    """Topology identical, floats within REL_TOL; returns True when bit-identical."""
    assert orc.status == 0
    n = len(orc.volume)
    assert np.array_equal(gpu.face_left, orc.face_left)
    assert np.array_equal(gpu.face_right, orc.face_right)
    assert np.array_equal(gpu.face_shift_code, orc.face_shift_code)
    if not faces_all:
        assert np.array_equal(gpu.cell_face_offset, orc.face_offset)
        assert np.array_equal(gpu.cell_face_count, orc.face_count)
        assert np.array_equal(gpu.cell_face_connections, orc.cell_face_connections)
    vscale = float(np.max(np.abs(orc.volume))) if n else 1.0
    lscale = vscale ** (1.0 / 3.0) if vscale > 0 else 1.0
    assert _rel_err(gpu.cell_volume, orc.volume, 1e-300) <= REL_TOL
    assert _rel_err(gpu.cell_centroid, orc.centroid, lscale) <= REL_TOL
    assert _rel_err(gpu.cell_safety_radius, orc.safety_radius, 1e-300) <= REL_TOL
    ascale = float(np.max(np.abs(orc.face_area))) if len(orc.face_area) else 1.0
    assert _rel_err(gpu.face_area, orc.face_area, ascale * 1e-6) <= REL_TOL
    assert _rel_err(gpu.face_centroid, orc.face_centroid, lscale) <= REL_TOL
    assert np.array_equal(gpu.face_normal, orc.face_normal)
    return (np.array_equal(gpu.cell_volume, orc.volume)
            and np.array_equal(gpu.cell_centroid, orc.centroid)
            and np.array_equal(gpu.face_area, orc.face_area)
            and np.array_equal(gpu.face_centroid, orc.face_centroid))
