"""Multi-rank (weak scaling) host logic of bench.py on CPU with gloo, world size 2.

Each rank tessellates its own independently seeded generator set (no collective on the
data path); the job time is the maximum over ranks and the throughput aggregates all
ranks' cells.  The per-rank tessellation here is the CPU oracle (no GPU needed).
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    import bench
    from meshless_voro_b200 import workloads as W
    from oracle import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        seed = bench.rank_seed(rank)
        w = W.poisson(3000, seed=seed, periodic=True)
        r = O.build(w["generators"], w["anchor"], w["width"], dim=3, periodic=True, nthreads=1)
        fake_ms = 10.0 * (rank + 1)                 # rank 1 is the slow one
        ms = bench.max_over_ranks(fake_ms, dist, torch.device("cpu"))
        value = bench.aggregate_cells_per_s(world, len(w["generators"]), ms)
        dist.barrier()
        out[rank] = (seed, r.status, float(r.volume.sum()), ms, value, float(w["generators"][0, 0]))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_weak_scaling_two_ranks():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True,
                       start_method="spawn")
    res = [out[r] for r in range(world)]
    seeds = [r[0] for r in res]
    assert len(set(seeds)) == world                      # independent inputs per rank
    assert res[0][5] != res[1][5]
    for seed, status, vsum, ms, value, _ in res:
        assert status == 0 and abs(vsum - 1.0) < 1e-12  # each rank's tessellation is complete
        assert ms == 20.0                                # max over ranks
        assert value == pytest.approx(world * 3000 / 0.020)


def test_single_process_identity():
    import bench
    assert bench.max_over_ranks(7.5, None, None) == 7.5
    assert bench.aggregate_cells_per_s(1, 1000, 1.0) == pytest.approx(1e6)


def test_batch_groups_split_by_generators():
    """bench.py's batched workload: consecutive groups of at most `cap` generators, a job
    larger than cap alone, order and membership kept."""
    import sys
    sys.path.insert(0, ROOT)
    import bench
    sizes = [5, 3, 9, 2, 2, 20, 1, 4]
    jobs = [dict(generators=np.zeros((k, 3)), tag=i) for i, k in enumerate(sizes)]
    groups = bench.batch_groups(jobs, cap=10)
    assert [j["tag"] for g in groups for j in g] == list(range(len(sizes)))
    for g in groups:
        total = sum(len(j["generators"]) for j in g)
        assert total <= 10 or len(g) == 1
    assert [[j["tag"] for j in g] for g in groups] == [[0, 1], [2], [3, 4], [5], [6, 7]]
