"""The C-ABI library loads and exports every entry point include/mvgpu.h declares.

Runs without a GPU: no compute calls, only loading, symbol lookup and the
device-free entry points.
"""
import ctypes as C
import os
import re

import pytest

from meshless_voro_b200 import _native as N
from meshless_voro_b200 import build as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "mvgpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mv_[a-z_0-9]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    B.build()
    return N.lib()


def test_header_symbols_match_binding():
    assert declared_symbols() == sorted(N.EXPORTED)


def test_every_declared_symbol_is_exported(lib):
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_strerror_and_version(lib):
    for code in range(0, 9):
        assert lib.mv_strerror(code)
    assert b"sm_100a" in lib.mv_version()


def test_options_default(lib):
    o = N.Options()
    lib.mv_options_default(C.byref(o))
    assert o.precision == N.MV_PRECISION_FILTERED
    assert o.face_mode == N.MV_FACES_OWNED


def test_shift_from_code(lib):
    w = (C.c_double * 3)(2.0, 3.0, 5.0)
    out = (C.c_double * 3)()
    # m = (1, -1, 0): shift = (w0, -w1, -0.0)
    code = (1 + 1) + 3 * (-1 + 1) + 9 * (0 + 1)
    lib.mv_shift_from_code(code, w, out)
    assert list(out) == [2.0, -3.0, 0.0]
    assert str(out[2]) == "-0.0"


def test_library_built_for_sm100a():
    assert "arch=compute_100a,code=sm_100a" in " ".join(B.NVCC_FLAGS)
    assert "--fmad=false" in B.NVCC_FLAGS


def test_no_device_is_reported_not_faked(lib):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    h = C.c_void_p()
    assert lib.mv_context_create(-1, C.byref(h)) == N.MV_ERR_NO_DEVICE


def test_batch_descriptor_layout():
    """mv_job / mv_batch_voronoi as the header lays them out, and the concatenated inputs
    batch_inputs hands to mv_context_build_batch."""
    assert C.sizeof(N.Job) == 8 + 48 + 16
    assert N.Job.dimensionality.offset == 56 and N.Job.has_mask.offset == 64
    assert C.sizeof(N.BatchVoronoi) == 4 * 8 + 3 * 8 + 12 * 8 + 2 * 8
    import numpy as np
    from meshless_voro_b200.voronoi import batch_inputs
    rng = np.random.default_rng(0)
    jobs = [dict(generators=rng.uniform(size=(5, 3)), anchor=[0, 0, 0], width=[1, 1, 1],
                 dimensionality=3, periodic=True),
            dict(generators=np.zeros((0, 3)), anchor=[1, 2, 3], width=[2, 2, 2],
                 dimensionality=2, periodic=False),
            dict(generators=rng.uniform(size=(4, 3)), anchor=[0, 0, 0], width=[1, 1, 1],
                 dimensionality=1, periodic=False, mask=[True, False, True, True])]
    g, m, d = batch_inputs(jobs)
    assert g.shape == (9, 3) and g.flags.c_contiguous
    assert np.array_equal(g[5:], jobs[2]["generators"])
    assert m.dtype == np.uint8 and list(m) == [1] * 5 + [1, 0, 1, 1]
    assert [x.n for x in d] == [5, 0, 4] and [x.has_mask for x in d] == [0, 0, 1]
    assert list(d[1].anchor) == [1, 2, 3] and d[1].dimensionality == 2 and d[1].periodic == 0
    g2, m2, _ = batch_inputs(jobs[:2])
    assert m2 is None and g2.shape == (5, 3)


def test_batch_workload_shape():
    """The batched configuration: sizes, dimensionality and mask mix as specified."""
    import numpy as np
    from meshless_voro_b200 import workloads as W
    jobs = W.batch_jobs(njobs=200, seed=9, nmin=50, nmax=2000)
    n = np.array([len(j["generators"]) for j in jobs])
    assert len(jobs) == 200 and n.min() >= 1 and n.max() <= 2000 * 1.2
    assert 0.6 < np.mean([j["dimensionality"] == 3 for j in jobs]) < 0.95
    for j in jobs:
        g, a, w = j["generators"], j["anchor"], j["width"]
        assert np.all(g >= a - 1e-12) and np.all(g <= a + w + 1e-12)
        assert np.all((w >= 0.5) & (w <= 2.0))
        if j["mask"] is not None:
            assert j["mask"].shape == (len(g),)


def test_batch_result_split():
    """batch_arrays splits a concatenated batch result by its per-tessellation offsets
    (no GPU: the result is assembled in host memory)."""
    import numpy as np
    from meshless_voro_b200.voronoi import batch_arrays, batch_inputs
    rng = np.random.default_rng(1)
    jobs = [dict(generators=rng.uniform(size=(3, 3)), anchor=[0, 0, 0], width=[1, 1, 1],
                 dimensionality=3, periodic=True),
            dict(generators=rng.uniform(size=(2, 3)), anchor=[0, 0, 0], width=[2, 2, 2],
                 dimensionality=2, periodic=False, mask=[True, False])]
    g, m, descs = batch_inputs(jobs)
    n, F, Cn = 5, 7, 9
    keep = []

    def buf(a):
        a = np.ascontiguousarray(a)
        keep.append(a)
        return a.ctypes.data_as(C.c_void_p)

    bv = N.BatchVoronoi()
    bv.n_jobs, bv.n_cells, bv.n_faces, bv.n_connections = 2, n, F, Cn
    offs = [(C.c_int64 * 3)(0, 3, 5), (C.c_int64 * 3)(0, 4, 7), (C.c_int64 * 3)(0, 6, 9)]
    bv.job_cell_offset, bv.job_face_offset, bv.job_connection_offset = [
        C.cast(o, C.POINTER(C.c_int64)) for o in offs]
    bv.cell_volume = buf(np.arange(n, dtype=np.float64))
    bv.cell_centroid = buf(np.arange(3 * n, dtype=np.float64))
    bv.cell_safety_radius = buf(np.ones(n))
    bv.cell_face_offset = buf(np.array([0, 2, 4, 0, 2], dtype=np.int64))
    bv.cell_face_count = buf(np.array([2, 2, 2, 2, 1], dtype=np.int32))
    bv.face_left = buf(np.array([0, 0, 1, 2, 0, 0, 1], dtype=np.int32))
    bv.face_right = buf(np.array([1, 2, 2, -1, 1, -1, -1], dtype=np.int32))
    bv.face_area = buf(np.arange(F, dtype=np.float64))
    bv.face_centroid = buf(np.zeros(3 * F))
    bv.face_normal = buf(np.zeros(3 * F))
    bv.face_shift_code = buf(np.full(F, 13, dtype=np.uint8))
    bv.cell_face_connections = buf(np.array([0, 1, 0, 2, 1, 3, 0, 1, 2], dtype=np.int32))
    a, b = batch_arrays(bv, descs, g, m)
    assert a.n_cells == 3 and b.n_cells == 2
    assert list(a.cell_volume) == [0, 1, 2] and list(b.cell_volume) == [3, 4]
    assert list(a.face_area) == [0, 1, 2, 3] and list(b.face_area) == [4, 5, 6]
    assert list(b.face_left) == [0, 0, 1] and list(b.face_right) == [1, -1, -1]
    assert list(a.cell_face_connections) == [0, 1, 0, 2, 1, 3]
    assert list(b.cell_face_connections) == [0, 1, 2]
    assert list(b.cell_face_offset) == [0, 2]
    assert b.dimensionality == 2 and not b.periodic and list(b.width) == [2, 2, 2]
    # 2D: z of the generator zeroed; the masked-out cell's location is zero
    assert b.cell_loc[0, 2] == 0.0 and np.all(b.cell_loc[1] == 0.0)
    assert np.array_equal(a.cell_loc, jobs[0]["generators"])
