"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

Topology -- faces (left, right, shift), their order, and the cell -> face CSR -- must
be identical.  Floating-point outputs must agree within 1e-12 relative to the
cell's scale; since the kernel keeps the reference's operation order they are
expected to be bit-identical, which is checked separately.
"""
import json
import math
import os
import zlib

import numpy as np
import pytest

import meshless_voro_b200 as mv
from meshless_voro_b200 import workloads as W
from meshless_voro_b200._native import MV_FACES_ALL, MV_FACES_OWNED, MvError
from voronoi_checks import REL_TOL, compare, consistency_check  # noqa: F401

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def _case(name):
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    if name == "single":
        return dict(generators=[[0.5, 0.5, 0.5]], anchor=[0, 0, 0], width=[1, 1, 1], dim=3, periodic=False)
    if name == "two":
        return dict(generators=[[0.3, 0.4, 0.25], [0.7, 0.6, 0.75]], anchor=[0, 0, 0], width=[1, 1, 1], dim=3, periodic=False)
    if name == "five_2d":
        d = math.sqrt(0.1)
        g = [[0.5, 0.5, 0.5], [0.5 - d, 0.5 - d, 0.5], [0.5 - d, 0.5 + d, 0.5], [0.5 + d, 0.5 + d, 0.5], [0.5 + d, 0.5 - d, 0.5]]
        return dict(generators=g, anchor=[0, 0, 0], width=[1, 1, 1], dim=2, periodic=False)
    if name == "four_2d_periodic":
        g = [[0.4, 0.3, 0], [1.6, 0.2, 0], [0.6, 0.8, 0], [1.4, 0.7, 0]]
        return dict(generators=g, anchor=[0, 0, 0], width=[2, 1, 1], dim=2, periodic=True)
    if name == "lattice4_rect":
        return dict(generators=W.perturbed_grid([0, 0, 0], [1, 1, 1], 4, 0.0, None), anchor=[0, 0, 0], width=[1, 1, 1], dim=3, periodic=False)
    if name == "lattice12_periodic":
        return dict(generators=W.perturbed_grid([0, 0, 0], [1, 1, 1], 12, 0.0, None), anchor=[0, 0, 0], width=[1, 1, 1], dim=3, periodic=True)
    if name == "jitter16_rect":
        return dict(generators=W.perturbed_grid([0, 0, 0], [1, 1, 1], 16, 0.5, rng), anchor=[0, 0, 0], width=[1, 1, 1], dim=3, periodic=False)
    if name == "grid15_w2":
        return dict(generators=W.perturbed_grid([0, 0, 0], [2, 2, 2], 15, 0.95, rng), anchor=[0, 0, 0], width=[2, 2, 2], dim=3, periodic=False)
    if name == "poisson20k_periodic":
        return dict(generators=rng.uniform(0, 1, (20000, 3)), anchor=[0, 0, 0], width=[1, 1, 1], dim=3, periodic=True)
    if name == "poisson5k_rect_aniso":
        g = rng.uniform(0, 1, (5000, 3)) * [3.0, 1.0, 0.5] + [-1.0, 2.0, 0.25]
        return dict(generators=g, anchor=[-1.0, 2.0, 0.25], width=[3.0, 1.0, 0.5], dim=3, periodic=False)
    if name == "small_periodic_17":
        return dict(generators=rng.uniform(0, 1, (17, 3)), anchor=[0, 0, 0], width=[1, 1, 1], dim=3, periodic=True)
    if name == "plane25_periodic_2d":
        return dict(generators=W.perturbed_plane([2, 2, 2], [2, 2, 1], 25, 0.95, rng), anchor=[2, 2, 2], width=[2, 2, 1], dim=2, periodic=True)
    if name == "poisson_2d_rect":
        return dict(generators=rng.uniform(0, 1, (3000, 3)), anchor=[0, 0, 0], width=[1, 1, 1], dim=2, periodic=False)
    if name == "line_1d_periodic":
        return dict(generators=rng.uniform(0, 1, (200, 3)), anchor=[0, 0, 0], width=[1, 1, 1], dim=1, periodic=True)
    if name == "non_perturbed_z":
        fx = json.load(open(os.path.join(HERE, "golden", "non_perturbed_z.json")))
        return dict(generators=fx["generators"], anchor=fx["anchor"], width=fx["width"], dim=3, periodic=False)
    if name == "clustered30k_periodic":
        return dict(generators=W.clustered(30000, 60, seed=11)["generators"], anchor=[0, 0, 0],
                    width=[1, 1, 1], dim=3, periodic=True)
    if name == "clustered20k_rect":
        return dict(generators=W.clustered(20000, 40, seed=12)["generators"], anchor=[0, 0, 0],
                    width=[1, 1, 1], dim=3, periodic=False)
    if name == "clustered_2d_periodic":
        return dict(generators=W.clustered(12000, 30, seed=13, dim=2)["generators"],
                    anchor=[0, 0, 0], width=[1, 1, 1], dim=2, periodic=True)
    if name == "clump6k_in_3k_periodic":
        # a compact clump in a sparse background: the safety radius of every cell on
        # the clump's surface takes in the whole clump (more than either staged list)
        g = np.concatenate([rng.uniform(0, 1, (3000, 3)),
                            np.mod([0.37, 0.52, 0.61] + 1e-3 * rng.standard_normal((6000, 3)), 1.0)])
        return dict(generators=g, anchor=[0, 0, 0], width=[1, 1, 1], dim=3, periodic=True)
    if name == "degenerate_2e15":
        g = W.perturbed_grid([0, 0, 0], [2e15] * 3, 10, 0.0, None)
        g[42] = 1e14 * np.array([1.00007490802, 9.00019014286, 5.00014639879])
        return dict(generators=g, anchor=[0, 0, 0], width=[2e15] * 3, dim=3, periodic=False)
    raise KeyError(name)


CASES = ["single", "two", "five_2d", "four_2d_periodic", "lattice4_rect", "lattice12_periodic",
         "jitter16_rect", "grid15_w2", "poisson20k_periodic", "poisson5k_rect_aniso",
         "small_periodic_17", "plane25_periodic_2d", "poisson_2d_rect", "line_1d_periodic",
         "non_perturbed_z", "degenerate_2e15", "clustered30k_periodic", "clustered20k_rect",
         "clustered_2d_periodic", "clump6k_in_3k_periodic"]


# the staged pipeline runs in small chunks so that every case spans several of them
PIPELINES = {"fused": dict(pipeline="fused"), "staged": dict(pipeline="staged", chunk_cells=997)}


@pytest.mark.parametrize("pipeline", ["fused", "staged"])
@pytest.mark.parametrize("precision", ["fp64", "filtered"])
@pytest.mark.parametrize("name", CASES)
def test_parity_full_build(gpu_ctx, oracle, name, precision, pipeline):
    c = _case(name)
    orc = oracle.build(c["generators"], c["anchor"], c["width"], dim=c["dim"], periodic=c["periodic"])
    gpu = gpu_ctx.build_arrays(c["generators"], None, c["anchor"], c["width"], c["dim"],
                               c["periodic"], precision=precision, **PIPELINES[pipeline])
    bit_identical = compare(gpu, orc)
    assert bit_identical, "expected bit-identical integrals"


@pytest.mark.parametrize("pipeline", ["fused", "staged"])
@pytest.mark.parametrize("precision", ["fp64", "filtered"])
@pytest.mark.parametrize("name", ["grid15_w2", "poisson20k_periodic", "plane25_periodic_2d"])
def test_parity_partial(gpu_ctx, oracle, name, precision, pipeline):
    c = _case(name)
    n = len(c["generators"])
    rng = np.random.default_rng(7)
    for mask in (rng.uniform(size=n) < 0.25, np.eye(1, n, n // 2, dtype=bool)[0]):
        orc = oracle.build(c["generators"], c["anchor"], c["width"], dim=c["dim"],
                           periodic=c["periodic"], mask=mask)
        gpu = gpu_ctx.build_arrays(c["generators"], mask, c["anchor"], c["width"], c["dim"],
                                   c["periodic"], precision=precision, **PIPELINES[pipeline])
        assert compare(gpu, orc)
        assert np.all(gpu.cell_volume[~mask] == 0.0)


@pytest.mark.parametrize("pipeline", ["fused", "staged"])
@pytest.mark.parametrize("name", ["grid15_w2", "poisson20k_periodic", "plane25_periodic_2d"])
def test_parity_all_faces_integrator(gpu_ctx, oracle, name, pipeline):
    """compute_face_integrals (non-symmetric): every face of every cell."""
    c = _case(name)
    orc = oracle.build(c["generators"], c["anchor"], c["width"], dim=c["dim"],
                       periodic=c["periodic"], flags=oracle.FACES_ALL | oracle.NO_CSR)
    gpu = gpu_ctx.build_arrays(c["generators"], None, c["anchor"], c["width"], c["dim"],
                               c["periodic"], face_mode=MV_FACES_ALL, **PIPELINES[pipeline])
    assert compare(gpu, orc, faces_all=True)


@pytest.mark.parametrize("precision", ["fp64", "filtered"])
def test_staged_retry_and_stats(gpu_ctx, oracle, precision):
    """A small initial radius sends many cells to the fused retry pass; the result and
    the per-cell counters must not depend on which kernel built a cell."""
    c = _case("poisson20k_periodic")
    orc = oracle.build(c["generators"], c["anchor"], c["width"], dim=3, periodic=True)
    stats = {}
    for pipe, kw in (("fused", dict(pipeline="fused")),
                     ("staged", dict(pipeline="staged", chunk_cells=4096, initial_radius=1.6))):
        gpu = gpu_ctx.build_arrays(c["generators"], None, c["anchor"], c["width"], 3, True,
                                   precision=precision, **kw)
        assert compare(gpu, orc)
        stats[pipe] = gpu_ctx.last_stats()
    assert stats["staged"]["staged_retries"] + stats["staged"]["staged_wide"] > 0
    assert stats["fused"]["staged_retries"] == 0 and stats["fused"]["staged_wide"] == 0
    for k in ("cells_built", "neighbours_clipped", "planes_added", "exact_tests", "serial_rings"):
        assert stats["staged"][k] == stats["fused"][k], k


@pytest.mark.parametrize("precision", ["filtered", "fp64"])
def test_staged_rounds_and_fused_fallback(gpu_ctx, oracle, precision):
    """Cells around a compact clump need more neighbours than the first staged list
    (the wide round takes them) and than the wide list (the fused kernel's staged big
    shells take them); every cell must come out as the oracle builds it."""
    c = _case("clump6k_in_3k_periodic")
    orc = oracle.build(c["generators"], c["anchor"], c["width"], dim=3, periodic=True)
    gpu = gpu_ctx.build_arrays(c["generators"], None, c["anchor"], c["width"], 3, True,
                               precision=precision, pipeline="staged", chunk_cells=2048)
    assert compare(gpu, orc)
    st = gpu_ctx.last_stats()
    assert st["staged_wide"] > 0 and st["staged_retries"] > 0
    fused = gpu_ctx.build_arrays(c["generators"], None, c["anchor"], c["width"], 3, True,
                                 precision=precision, pipeline="fused")
    assert compare(fused, orc)
    sf = gpu_ctx.last_stats()
    for k in ("cells_built", "neighbours_clipped", "planes_added", "exact_tests", "serial_rings"):
        assert st[k] == sf[k], k


def test_reference_api_kats(gpu_ctx):
    """The reference's own unit tests, run through the mirrored API on the GPU."""
    v = mv.Voronoi.build([[0.5, 0.5, 0.5]], [0, 0, 0], [1, 1, 1], mv.Dimensionality.ThreeD, False,
                         context=gpu_ctx)
    assert abs(v.cells()[0].volume() - 1.0) < 1e-15
    for n in (2, 3, 4):
        g = W.perturbed_grid([0, 0, 0], [1, 1, 1], n, 0.0, None)
        v = mv.Voronoi.build(g, [0, 0, 0], [1, 1, 1], 3, False, context=gpu_ctx)
        assert np.allclose(v.arrays.cell_volume, 1.0 / n ** 3, rtol=0, atol=1e-15)
    g = W.perturbed_grid([0, 0, 0], [2, 2, 2], 15, 0.95, np.random.default_rng(3))
    v = mv.Voronoi.build(g, [0, 0, 0], [2, 2, 2], 3, False, context=gpu_ctx)
    a = v.arrays
    consistency_check(a, 3, [2, 2, 2])
    # neighbour_ids of a cell are the other side of its internal faces
    cell = v.cells()[100]
    ids = sorted(cell.neighbour_ids())
    assert len(ids) == cell.face_count() - sum(1 for f in cell.faces() if f.is_boundary())


@pytest.mark.parametrize("pipeline", ["fused", "staged"])
def test_duplicate_generators_raise(gpu_ctx, pipeline):
    """convex_cell.rs:325-342 panics on a duplicate; the library names a duplicated cell."""
    g = [[0.7, 0.7, 0.7], [0.2, 0.2, 0.2], [0.4, 0.5, 0.6], [0.2, 0.2, 0.2]]
    with pytest.raises(MvError) as e:
        gpu_ctx.build_arrays(g, None, [0, 0, 0], [1, 1, 1], 3, False, **PIPELINES[pipeline])
    assert e.value.status == 2
    assert e.value.error_cell in (1, 3)


def test_empty_input(gpu_ctx):
    a = gpu_ctx.build_arrays(np.zeros((0, 3)), None, [0, 0, 0], [1, 1, 1], 3, False)
    assert a.n_cells == 0 and len(a.face_left) == 0


def test_plate_lattice_wide_round_ties(gpu_ctx, oracle):
    """An exact lattice of thin plates (16 x 16 x 256 in the periodic unit box, 65,536
    cells): the probe chunk selects the clip kernel's box form (every band test is a
    box-corner zero), no first shell closes a cell (they are 16 times wider than
    thick), and every wide-round shell is full of equal squared distances, so the wide
    round's equal-key fallback (the shell gathered again and fully sorted) builds them."""
    i = (np.arange(16) + 0.5) / 16
    k = (np.arange(256) + 0.5) / 256
    g = np.stack(np.meshgrid(i, i, k, indexing="ij"), -1).reshape(-1, 3)
    orc = oracle.build(g, [0, 0, 0], [1, 1, 1], dim=3, periodic=True)
    for precision in ("filtered", "fp64"):
        gpu = gpu_ctx.build_arrays(g, None, [0, 0, 0], [1, 1, 1], 3, True, precision=precision)
        assert compare(gpu, orc), "expected bit-identical integrals"
        st = gpu_ctx.last_stats()
        assert st["staged_wide"] > 0 and st["exact_tests"] > 0, st
