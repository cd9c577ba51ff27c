"""GPU parity of batch builds (mv_context_build_batch): every tessellation of a batch
comes out exactly as the oracle builds it alone, and exactly as a single GPU build of
it -- faces, their order, the CSR and every floating-point value, bit for bit.
"""
import numpy as np
import pytest

import meshless_voro_b200 as mv
from meshless_voro_b200 import workloads as W
from meshless_voro_b200._native import MV_FACES_ALL, MV_FACES_OWNED, MvError
from voronoi_checks import compare

pytestmark = pytest.mark.gpu


def _mixed_jobs():
    rng = np.random.default_rng(77)
    jobs = [
        dict(generators=rng.uniform(0, 1, (3000, 3)), anchor=[0, 0, 0], width=[1, 1, 1],
             dimensionality=3, periodic=True),
        dict(generators=W.perturbed_grid([-1, 0.5, 2], [2, 1, 0.5], 11, 0.5, rng),
             anchor=[-1, 0.5, 2], width=[2, 1, 0.5], dimensionality=3, periodic=False),
        dict(generators=np.zeros((0, 3)), anchor=[0, 0, 0], width=[1, 1, 1], dimensionality=3,
             periodic=True),
        dict(generators=[[0.25, 0.5, 0.75]], anchor=[0, 0, 0], width=[1, 1, 1],
             dimensionality=3, periodic=False),
        dict(generators=W.perturbed_plane([0, 0, 0], [1.5, 1, 1], 30, 0.9, rng),
             anchor=[0, 0, 0], width=[1.5, 1, 1], dimensionality=2, periodic=True),
        dict(generators=rng.uniform(0, 1, (1200, 3)), anchor=[0, 0, 0], width=[1, 1, 1],
             dimensionality=2, periodic=False),
        dict(generators=rng.uniform(0, 1, (400, 3)), anchor=[0, 0, 0], width=[1, 1, 1],
             dimensionality=1, periodic=True),
        dict(generators=rng.uniform(0, 2, (2500, 3)), anchor=[0, 0, 0], width=[2, 2, 2],
             dimensionality=3, periodic=True, mask=rng.uniform(size=2500) < 0.7),
        dict(generators=W.clustered(6000, 12, seed=31)["generators"], anchor=[0, 0, 0],
             width=[1, 1, 1], dimensionality=3, periodic=True),
        dict(generators=W.perturbed_grid([0, 0, 0], [1, 1, 1], 8, 0.0, None), anchor=[0, 0, 0],
             width=[1, 1, 1], dimensionality=3, periodic=True),
    ]
    return jobs


def _oracle(oracle, j, faces_all=False):
    return oracle.build(np.asarray(j["generators"], dtype=np.float64).reshape(-1, 3), j["anchor"],
                        j["width"], dim=j["dimensionality"], periodic=j["periodic"],
                        mask=j.get("mask"), flags=oracle.FACES_ALL if faces_all else 0)


def _same(a, b):
    for k in ("cell_volume", "cell_centroid", "cell_safety_radius", "face_left", "face_right",
              "face_area", "face_centroid", "face_normal", "face_shift_code",
              "cell_face_offset", "cell_face_count", "cell_face_connections"):
        x, y = getattr(a, k), getattr(b, k)
        if x is None or y is None:
            assert x is None and y is None, k
        else:
            assert np.array_equal(x, y), k


@pytest.mark.parametrize("precision", ["filtered", "fp64"])
def test_batch_matches_oracle_and_single_builds(gpu_ctx, oracle, precision):
    jobs = _mixed_jobs()
    res = gpu_ctx.build_batch(jobs, precision=precision, chunk_cells=4096)
    assert len(res) == len(jobs)
    st = gpu_ctx.last_stats()
    assert st["cells_built"] == sum(int(np.sum(j["mask"])) if j.get("mask") is not None
                                    else len(j["generators"]) for j in jobs)
    for j, r in zip(jobs, res):
        if len(j["generators"]) == 0:
            assert r.n_cells == 0 and len(r.face_left) == 0
            continue
        assert compare(r, _oracle(oracle, j))
        single = gpu_ctx.build_arrays(j["generators"], j.get("mask"), j["anchor"], j["width"],
                                      j["dimensionality"], j["periodic"], precision=precision)
        _same(r, single)


def test_batch_faces_all(gpu_ctx, oracle):
    jobs = _mixed_jobs()[:2] + _mixed_jobs()[4:6]
    res = gpu_ctx.build_batch(jobs, face_mode=MV_FACES_ALL)
    for j, r in zip(jobs, res):
        assert r.cell_face_connections is None
        assert compare(r, _oracle(oracle, j, faces_all=True), faces_all=True)


def test_batch_of_one_equals_single(gpu_ctx):
    j = _mixed_jobs()[0]
    (r,) = gpu_ctx.build_batch([j])
    single = gpu_ctx.build_arrays(j["generators"], None, j["anchor"], j["width"], 3, True)
    _same(r, single)


def test_batch_error_names_job_and_cell(gpu_ctx):
    """A duplicate generator (the reference panics, convex_cell.rs:325-342) is reported
    with its tessellation and its local index."""
    jobs = _mixed_jobs()[:2]
    g = np.asarray(jobs[1]["generators"]).copy()
    g[17] = g[5]
    jobs[1] = dict(jobs[1], generators=g)
    with pytest.raises(MvError) as e:
        gpu_ctx.build_batch(jobs)
    assert e.value.error_job == 1
    assert e.value.error_cell in (5, 17)
    # the context stays usable
    (r,) = gpu_ctx.build_batch(jobs[:1])
    assert r.n_cells == 3000


def test_batch_generated_workload(gpu_ctx, oracle):
    """A small draw of the batched configuration's generator, job by job against the
    oracle (lattices, partial masks, 2D and 3D, periodic and rectangular)."""
    jobs = W.batch_jobs(njobs=24, seed=13, nmin=200, nmax=4000)
    res = gpu_ctx.build_batch(jobs, chunk_cells=2048)
    for j, r in zip(jobs, res):
        assert compare(r, _oracle(oracle, j))
