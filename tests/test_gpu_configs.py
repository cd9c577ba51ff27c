"""GPU parity at the benchmark configurations' own sizes.

* C1 -- 32^3 lattice jittered by U(+-0.25 spacing), rectangular unit box: compared
  with the oracle in full (every face, the CSR, every value).
* C2 -- 64^3 exact lattice, periodic unit box: every Voronoi vertex is shared by eight
  co-spherical generators, so the f64 clip test is undecided everywhere and the exact
  integer predicate decides (the reference's perfect-grid case); compared in full, and
  the build must have run exact tests.
* C3 -- 256^3 i.i.d. uniform, periodic, and C4 -- 8,388,608 points, half of them in
  2000 Gaussian clumps, periodic: a seeded sample of cells against the oracle's
  partial build of the same cells (the comparison of voronoi.rs:1052-1085), and the
  volume closure over all cells.
* C5 -- the 4096-tessellation uneven batch: the first batch build of the benchmark's
  grouping, a sample of its tessellations compared in full.

Topology is bit-exact; the integrals must lie within 1e-12 relative of the oracle's
(REL_TOL), and since the kernels keep the reference's operation order they are
expected to be bit-identical, which is asserted too.  Volumes must sum to the box
volume within 1e-12 relative (exactly rounded sum).
"""
import types

import numpy as np
import pytest

from meshless_voro_b200 import workloads as W
from meshless_voro_b200.voronoi import batch_inputs, device_tensors
from voronoi_checks import REL_TOL, compare

pytestmark = pytest.mark.gpu

SEED = 3  # the benchmark's seed for these workloads


def _full(gpu_ctx, oracle, w, precision, pipeline):
    orc = oracle.build(w["generators"], w["anchor"], w["width"], dim=w["dimensionality"],
                       periodic=w["periodic"])
    gpu = gpu_ctx.build_arrays(w["generators"], None, w["anchor"], w["width"],
                               w["dimensionality"], w["periodic"], precision=precision,
                               pipeline=pipeline)
    assert compare(gpu, orc), "expected bit-identical integrals"
    box = float(np.prod(w["width"][:w["dimensionality"]]))
    assert abs(np.sum(gpu.cell_volume) - box) <= 1e-12 * box
    return gpu_ctx.last_stats()


@pytest.mark.parametrize("pipeline", ["auto", "staged"])
@pytest.mark.parametrize("precision", ["filtered", "fp64"])
def test_c1_jittered_lattice_32_full(gpu_ctx, oracle, precision, pipeline):
    _full(gpu_ctx, oracle, W.jittered_lattice_32(SEED), precision, pipeline)


@pytest.mark.parametrize("pipeline", ["auto", "staged", "fused"])
@pytest.mark.parametrize("precision", ["filtered", "fp64"])
def test_c2_exact_lattice_64_full(gpu_ctx, oracle, precision, pipeline):
    st = _full(gpu_ctx, oracle, W.exact_lattice(64), precision, pipeline)
    assert st["exact_tests"] > 0
    assert st["cells_built"] == 64 ** 3
    if pipeline == "auto":
        # every band test of the lattice is a box-corner zero, which the staged clip
        # kernel decides itself: the staged pipeline builds the lattice
        assert st["ms_shell"] > 0 and st["staged_retries"] < 0.1 * 64 ** 3


_SAMPLES = {}


def _oracle_sample(parity, key, w, idx):
    if key not in _SAMPLES:
        _SAMPLES[key] = parity.oracle_sample(w, idx)
    return _SAMPLES[key]


def _sampled(gpu_ctx, w, key, frac, precision):
    import torch
    from oracle import parity
    n = len(w["generators"])
    g = torch.from_numpy(np.ascontiguousarray(w["generators"])).cuda()
    torch.cuda.synchronize()
    dv = gpu_ctx.build_device(g.data_ptr(), 0, n, w["anchor"], w["width"], w["dimensionality"],
                              w["periodic"], precision=precision,
                              stream=torch.cuda.current_stream().cuda_stream)
    t = device_tensors(dv)
    idx = parity.sample_cells(n, frac, seed=SEED + 100)
    gs = parity.device_sample(t, idx)
    vol = t["cell_volume"].cpu().numpy()
    res = parity.compare_sample(gs, _oracle_sample(parity, key, w, idx))
    assert res["topology_mismatched_cells"] == 0, res
    assert max(res["max_rel_err"].values()) <= REL_TOL, res
    assert res["bit_identical"], res
    cl = parity.closure(vol, w["width"], w["dimensionality"])
    assert cl["ok"], cl
    return gpu_ctx.last_stats()


@pytest.mark.parametrize("precision", ["filtered", "fp64"])
def test_c3_poisson_256_sampled(gpu_ctx, precision):
    w = W.poisson(256 ** 3, seed=SEED, periodic=True)
    st = _sampled(gpu_ctx, w, "c3", 0.005, precision)
    assert st["cells_built"] == 256 ** 3


@pytest.mark.parametrize("precision", ["filtered", "fp64"])
def test_c4_clustered_sampled(gpu_ctx, precision):
    w = W.clustered(8388608, 2000, seed=SEED)
    st = _sampled(gpu_ctx, w, "c4", 0.0025, precision)
    assert st["cells_built"] == 8388608


def test_c5_batch_sampled(gpu_ctx, oracle):
    import torch
    jobs = W.batch_jobs(njobs=4096, seed=SEED)
    # the benchmark's first batch build: consecutive jobs up to 2^25 generators
    grp, m = [], 0
    for j in jobs:
        if grp and m + len(j["generators"]) > (1 << 25):
            break
        grp.append(j)
        m += len(j["generators"])
    g, mask, descs = batch_inputs(grp)
    gd = torch.from_numpy(g).cuda()
    md = torch.from_numpy(mask).cuda() if mask is not None else None
    torch.cuda.synchronize()
    bv = gpu_ctx.build_batch_device(gd.data_ptr(), md.data_ptr() if md is not None else 0, descs,
                                    stream=torch.cuda.current_stream().cuda_stream)
    t = device_tensors(bv)
    co, fo, no = bv.job_cell_offset, bv.job_face_offset, bv.job_connection_offset
    rng = np.random.default_rng(SEED)
    pick = set(rng.choice(len(grp), size=min(6, len(grp)), replace=False).tolist())
    # make sure a partial build and a 2D tessellation are among them
    for cond in (lambda j: j.get("mask") is not None, lambda j: j["dimensionality"] == 2):
        k = next((i for i, j in enumerate(grp) if cond(j)), None)
        if k is not None:
            pick.add(k)
    for k in sorted(pick):
        j = grp[k]
        c0, c1, f0, f1, n0, n1 = co[k], co[k + 1], fo[k], fo[k + 1], no[k], no[k + 1]
        arr = types.SimpleNamespace(
            cell_volume=t["cell_volume"][c0:c1].cpu().numpy(),
            cell_centroid=t["cell_centroid"][c0:c1].cpu().numpy(),
            cell_safety_radius=t["cell_safety_radius"][c0:c1].cpu().numpy(),
            cell_face_offset=t["cell_face_offset"][c0:c1].cpu().numpy(),
            cell_face_count=t["cell_face_count"][c0:c1].cpu().numpy().astype(np.int64),
            face_left=t["face_left"][f0:f1].cpu().numpy().astype(np.int64),
            face_right=t["face_right"][f0:f1].cpu().numpy().astype(np.int64),
            face_area=t["face_area"][f0:f1].cpu().numpy(),
            face_centroid=t["face_centroid"][f0:f1].cpu().numpy(),
            face_normal=t["face_normal"][f0:f1].cpu().numpy(),
            face_shift_code=t["face_shift_code"][f0:f1].cpu().numpy().astype(np.int32),
            cell_face_connections=t["cell_face_connections"][n0:n1].cpu().numpy().astype(np.int64))
        orc = oracle.build(j["generators"], j["anchor"], j["width"], dim=j["dimensionality"],
                           periodic=j["periodic"], mask=j.get("mask"))
        assert compare(arr, orc), f"tessellation {k}: expected bit-identical integrals"
