"""mv_voronoi_build_noalloc: the build entry point that allocates nothing.

It serves callers that cannot call cudaMalloc (their device memory belongs to another
allocator, or they must avoid the implicit synchronisation of cudaMalloc/cudaFree):
all scratch lives in a fixed static device array inside the library and the caller
passes the input and output buffers.  These tests call it through the C ABI and
check it against the regular entry point (mv_context_build) on two calls in a row,
so the second call also proves that the scratch left by the first one does not leak
into its result.  The file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from meshless_voro_b200 import _native as N
from meshless_voro_b200 import workloads as W
from meshless_voro_b200.voronoi import make_options

pytestmark = pytest.mark.gpu
REL_TOL = 1e-12


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def noalloc_build(torch, g, anchor, width, dim, periodic, precision, mask=None,
                  face_mode=N.MV_FACES_OWNED, fcap=None, expect=N.MV_OK):
    """Caller-allocated device buffers (torch), then the no-alloc entry point."""
    dev = torch.device("cuda", 0)
    n = g.shape[0]
    fcap = 18 * n + 64 if fcap is None else fcap
    ccap = 2 * fcap
    gd = torch.from_numpy(np.ascontiguousarray(g)).to(dev)
    md = None
    if mask is not None:
        md = torch.from_numpy(np.ascontiguousarray(mask, dtype=np.bool_).view(np.uint8)).to(dev)
    buf = dict(
        cell_volume=torch.empty(n, dtype=torch.float64, device=dev),
        cell_centroid=torch.empty(n, 3, dtype=torch.float64, device=dev),
        cell_safety_radius=torch.empty(n, dtype=torch.float64, device=dev),
        face_left=torch.empty(fcap, dtype=torch.int32, device=dev),
        face_right=torch.empty(fcap, dtype=torch.int32, device=dev),
        face_area=torch.empty(fcap, dtype=torch.float64, device=dev),
        face_centroid=torch.empty(fcap, 3, dtype=torch.float64, device=dev),
        face_normal=torch.empty(fcap, 3, dtype=torch.float64, device=dev),
        face_shift_code=torch.empty(fcap, dtype=torch.uint8, device=dev),
    )
    if face_mode == N.MV_FACES_OWNED:
        buf.update(cell_face_offset=torch.empty(n, dtype=torch.int64, device=dev),
                   cell_face_count=torch.empty(n, dtype=torch.int32, device=dev),
                   cell_face_connections=torch.empty(ccap, dtype=torch.int32, device=dev))
    out = N.DeviceVoronoi()
    for k, t in buf.items():
        setattr(out, k, t.data_ptr())
    opts = make_options(precision, face_mode=face_mode,
                        stream=torch.cuda.current_stream(dev).cuda_stream)
    a = np.ascontiguousarray(np.asarray(anchor, dtype=np.float64))
    w = np.ascontiguousarray(np.asarray(width, dtype=np.float64))
    rc = N.lib().mv_voronoi_build_noalloc(C.c_void_p(gd.data_ptr()),
                                          C.c_void_p(md.data_ptr()) if md is not None else None,
                                          n, _dp(a), _dp(w), dim, int(periodic), C.byref(opts),
                                          C.byref(out), fcap, ccap)
    torch.cuda.synchronize(dev)
    if expect != N.MV_OK:
        assert rc == expect
        return out
    N.check(rc, out.error_cell)
    F, Cn = int(out.n_faces), int(out.n_connections)
    h = {k: t.cpu().numpy() for k, t in buf.items()}
    for k in ("face_left", "face_right", "face_area", "face_centroid", "face_normal", "face_shift_code"):
        h[k] = h[k][:F]
    if "cell_face_connections" in h:
        h["cell_face_connections"] = h["cell_face_connections"][:Cn]
    return h


def _close(a, b, scale):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.size == 0:
        return True
    return float(np.max(np.abs(a - b) / (np.abs(b) + scale))) <= REL_TOL


def check_against_regular(ctx, torch, g, anchor, width, dim, periodic, precision, mask=None,
                          face_mode=N.MV_FACES_OWNED):
    h = noalloc_build(torch, g, anchor, width, dim, periodic, precision, mask, face_mode)
    r = ctx.build_arrays(g, mask, anchor, width, dim, periodic, precision=precision,
                         face_mode=face_mode)
    keys = ["face_left", "face_right", "face_shift_code"]
    if face_mode == N.MV_FACES_OWNED:
        keys += ["cell_face_offset", "cell_face_count", "cell_face_connections"]
    for k in keys:
        assert np.array_equal(np.asarray(h[k], dtype=np.int64), np.asarray(getattr(r, k), dtype=np.int64)), k
    vmax = float(np.max(np.abs(r.cell_volume)))
    lscale = vmax ** (1.0 / 3.0) if vmax > 0 else 1.0
    assert _close(h["cell_volume"], r.cell_volume, 1e-300)
    assert _close(h["cell_centroid"], r.cell_centroid, lscale)
    assert _close(h["cell_safety_radius"], r.cell_safety_radius, 1e-300)
    assert _close(h["face_area"], r.face_area, float(np.max(r.face_area)) * 1e-6)
    assert _close(h["face_centroid"], r.face_centroid, lscale)
    assert np.array_equal(h["face_normal"], r.face_normal)


@pytest.mark.parametrize("precision", ["filtered", "fp64"])
def test_noalloc_matches_regular_two_calls(gpu_ctx, precision):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(11)
    # first call: 3-D periodic Poisson
    g1 = rng.uniform(0.0, 1.0, size=(20000, 3))
    check_against_regular(gpu_ctx, torch, g1, [0, 0, 0], [1, 1, 1], 3, True, precision)
    # second call, smaller and different: the scratch still holds the first call's data
    g2 = W.perturbed_grid([0, 0, 0], [2, 1, 1], 12, 0.5, rng)
    check_against_regular(gpu_ctx, torch, g2, [0, 0, 0], [2, 1, 1], 3, False, precision)


def _inputs(kind, rng):
    if kind == "3d_periodic_max":
        # the largest set the entry point takes
        return rng.uniform(0, 1, (32768, 3)), [0, 0, 0], [1, 1, 1], 3, True
    if kind == "2d_rect":
        return rng.uniform(0, 1, (5000, 3)), [0, 0, 0], [1, 1, 1], 2, False
    if kind == "1d_periodic":
        return rng.uniform(0, 1, (700, 3)), [0, 0, 0], [1, 1, 1], 1, True
    if kind == "clustered_3d":
        # a compact clump: the shells of the cells around it do not fit shared memory
        g = np.concatenate([rng.uniform(0, 1, (3000, 3)),
                            np.mod([0.37, 0.52, 0.61] + 1e-3 * rng.standard_normal((6000, 3)), 1.0)])
        return g, [0, 0, 0], [1, 1, 1], 3, True
    raise KeyError(kind)


@pytest.mark.parametrize("masked", [False, True])
@pytest.mark.parametrize("face_mode", [N.MV_FACES_OWNED, N.MV_FACES_ALL])
@pytest.mark.parametrize("kind", ["3d_periodic_max", "2d_rect", "1d_periodic", "clustered_3d"])
def test_noalloc_dims_modes_masks(gpu_ctx, kind, face_mode, masked):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(5)
    g, a, w, dim, periodic = _inputs(kind, rng)
    mask = rng.uniform(size=len(g)) < 0.6 if masked else None
    check_against_regular(gpu_ctx, torch, g, a, w, dim, periodic, "filtered", mask, face_mode)


def test_noalloc_reports_needed_faces(gpu_ctx):
    """Too small an output: MV_ERR_CAPACITY, with the number of faces the build needs."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(9)
    g = rng.uniform(0, 1, (4000, 3))
    r = gpu_ctx.build_arrays(g, None, [0, 0, 0], [1, 1, 1], 3, True)
    out = noalloc_build(torch, g, [0, 0, 0], [1, 1, 1], 3, True, "filtered", fcap=100,
                        expect=N.MV_ERR_CAPACITY)
    assert int(out.n_faces) == len(r.face_left)
    # and a call with enough room right after still matches
    check_against_regular(gpu_ctx, torch, g, [0, 0, 0], [1, 1, 1], 3, True, "filtered")


def test_noalloc_rejects_oversize():
    a = np.zeros(3)
    w = np.ones(3)
    out = N.DeviceVoronoi()
    n = 32768 + 1  # MV_NOALLOC_MAX_GENERATORS + 1
    rc = N.lib().mv_voronoi_build_noalloc(C.c_void_p(1), None, n, _dp(a), _dp(w), 3, 0, None,
                                          C.byref(out), 0, 0)
    assert rc == N.MV_ERR_CAPACITY
