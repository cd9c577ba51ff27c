#!/usr/bin/env python
"""Benchmark: 3D Voronoi cells/s on B200 (meshless_voronoi per-cell construction path).

A step is one complete tessellation of the workload: generator prep + uniform grid,
cell construction (neighbour shells, clipping, exact predicates, integrals), face
ordering and the cell -> face CSR.  Default workload: 256^3 = 16,777,216 i.i.d.
uniform generators in the periodic unit box (seeded, synthetic).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision filtered|fp64]
                  [--workload poisson_256|lattice_64|jitter_32|grid_64|grid_64_p95|clustered|
                              batch_4096]
                  [--impl ours|reference]
                  [--pipeline auto|staged|fused]

The default pipeline runs the staged shell / clip / integral kernels; the plain FP64
comparison is the fused one-kernel-per-cell FP64 build of the same workload.

With N > 1 (torchrun, one process per GPU) every rank tessellates its own
independently seeded generator set (weak scaling, no collective on the data path);
value = all ranks' cells / max over ranks of the device time.

Outside the timed region the timed build is checked against the oracle (`parity` in
the JSON line: full comparison up to 2^20 cells, a seeded sample of cells above, the
volume closure over all cells; batches: sampled tessellations in full).  `e2e` runs the
same workload through mv_context_build with pinned host buffers, every result copied
back each step, on --e2e-contexts contexts (one host thread each) so copies of one build
overlap the kernels of another.  The reference arm builds every cell of the workload
once, split over the K steps.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "3D Voronoi cells/s on 1 B200: FP32-filtered batched vs plain FP64, exact topology"
HBM_PEAK_FALLBACK = 6650.0
# DRAM bytes (read + write) per cell of the clip kernel, from one ncu capture of the
# clip kernel on the 64^3 periodic Poisson case; traffic grows in proportion to the
# cells, so a launch's traffic is this figure times its cells.
CLIP_KERNEL_DRAM_BYTES_PER_CELL = 2026.0
# algorithmic bytes (generator read + cell outputs + owned faces + CSR entries)
BYTES_GEN, BYTES_CELL, BYTES_FACE, BYTES_CONN = 24, 40, 68, 4
# cells per chunk of the staged pipeline (library default)
CHUNK_CELLS = 1 << 20


def rank_seed(rank: int, base: int = 3) -> int:
    """Weak scaling: every rank tessellates its own independently seeded generator set."""
    return base + rank


def max_over_ranks(value: float, dist, device) -> float:
    """Slowest rank's time (the job's time); identity without a process group."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_cells_per_s(world: int, n_per_rank: int, ms_max: float) -> float:
    """Whole-job throughput: all ranks' cells over the slowest rank's time."""
    return world * n_per_rank / (ms_max * 1e-3)


def workload(name: str, seed: int):
    from meshless_voro_b200 import workloads as W
    if name == "poisson_256":
        w = W.poisson(256 ** 3, seed=seed, periodic=True)
        w["name"] = "poisson_256^3_periodic_unit_box"
    elif name == "lattice_64":
        w = W.exact_lattice(64)
    elif name == "jitter_32":
        w = W.jittered_lattice_32(seed)
    elif name == "grid_64":
        w = W.grid_example(64, 0.0)
    elif name == "grid_64_p95":
        w = W.grid_example(64, 0.95, seed)
    elif name == "clustered":
        w = W.clustered(8388608, 2000, seed=seed)
    elif name.startswith("clustered_"):
        w = W.clustered(int(name.split("_")[1]), 2000, seed=seed)
    elif name.startswith("poisson_"):
        n = int(name.split("_")[1]) ** 3
        w = W.poisson(n, seed=seed, periodic=True)
    else:
        raise SystemExit(f"unknown workload {name}")
    return w


BATCH_GROUP_CELLS = 1 << 25  # generators per batch build (device memory bound)
FULL_PARITY_CELLS = 1 << 20   # parity compares every cell up to this size, else a sample
L2_FLUSH_BYTES = 256 << 20    # inputs below this are timed step by step with L2 flushed


def batch_groups(jobs, cap=BATCH_GROUP_CELLS):
    """Consecutive groups of jobs with at most `cap` generators each (a job larger than
    cap forms its own group)."""
    groups, cur, m = [], [], 0
    for j in jobs:
        k = len(j["generators"])
        if cur and m + k > cap:
            groups.append(cur)
            cur, m = [], 0
        cur.append(j)
        m += k
    if cur:
        groups.append(cur)
    return groups


def cpu_baseline_batch(jobs, budget_s=12.0, threads=None):
    """The oracle on all host cores, one tessellation after another (as a caller of the
    reference loops over Voronoi::build), over the batch's first jobs for about
    budget_s seconds; cells/s extrapolated to the batch."""
    from oracle import oracle as O
    threads = threads or os.cpu_count()
    cells, t, k = 0, 0.0, 0
    for j in jobs:
        t0 = time.perf_counter()
        r = O.build(j["generators"], j["anchor"], j["width"], dim=j["dimensionality"],
                    periodic=j["periodic"], mask=j.get("mask"), nthreads=threads, flags=O.NO_CSR)
        assert r.status == 0
        t += time.perf_counter() - t0
        cells += len(j["generators"])
        k += 1
        if t >= budget_s:
            break
    return {"value": cells / t, "unit": "cells/s", "cores": threads, "kind": "port",
            "sample": f"the first {k} of the {len(jobs)} tessellations ({cells} cells, "
                      f"{t:.1f} s), one build per tessellation"}


def run_batch(args, rank, world):
    """Batched uneven tessellations: every step builds all jobs (in groups of at most
    BATCH_GROUP_CELLS generators, one mv_context_build_batch_device call each)."""
    import ctypes as C
    import torch
    import torch.distributed as dist
    import meshless_voro_b200 as mv
    from meshless_voro_b200 import _native as NN
    from meshless_voro_b200 import workloads as W
    from meshless_voro_b200.voronoi import batch_inputs

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", device_id=dev,
                                timeout=__import__("datetime").timedelta(seconds=300))
    njobs = int(args.workload.split("_")[1])
    jobs = W.batch_jobs(njobs=njobs, seed=rank_seed(rank))
    n = sum(len(j["generators"]) for j in jobs)
    groups, jobs_by_group = [], batch_groups(jobs)
    for grp in jobs_by_group:
        g, m, descs = batch_inputs(grp)
        gh = torch.from_numpy(g).pin_memory()
        mh = torch.from_numpy(m).pin_memory() if m is not None else None
        groups.append(dict(gh=gh, mh=mh, gd=gh.to(dev), md=mh.to(dev) if mh is not None else None,
                           descs=descs, n=len(g)))
    ctx = mv.Context(local)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream

    def step():
        stats, F, Cn = [], 0, 0
        for gr in groups:
            d_mask = gr["md"].data_ptr() if gr["md"] is not None else 0
            out = ctx.build_batch_device(gr["gd"].data_ptr(), d_mask, gr["descs"],
                                         precision=args.precision, stream=sp)
            F += int(out.n_faces)
            Cn += int(out.n_connections)
            stats.append(ctx.last_stats())
        return stats, F, Cn

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            r = fn()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return max_over_ranks(e0.elapsed_time(e1) / args.steps, dist, dev), r

    with ClockSampler(local) as clk:
        ms, (stats, F, Cn) = timed(step)
    clocks = clk.summary()
    value = aggregate_cells_per_s(world, n, ms)
    parity = None
    if rank == 0 and not args.no_parity:
        parity = parity_batch(ctx, groups, jobs_by_group, precision=args.precision, stream=sp)

    e2e = None
    if not args.no_e2e:
        # host buffers through mv_context_build_batch; the step's batch builds are split
        # over args.e2e_contexts contexts on as many host threads, so the result copy of
        # one batch build overlaps the kernels of the next
        nctx = max(1, min(args.e2e_contexts, len(groups)))
        ctxs = [ctx] + [mv.Context(local) for _ in range(nctx - 1)]
        streams = [stream] + [torch.cuda.Stream(dev) for _ in range(nctx - 1)]
        opts = [mv.voronoi.make_options(args.precision, stream=s_.cuda_stream) for s_ in streams]
        d2h_box = [0] * nctx
        errors = []

        def worker(i):
            try:
                for gi in range(i, len(groups), nctx):
                    gr = groups[gi]
                    bv = NN.BatchVoronoi()
                    rc = NN.lib().mv_context_build_batch(
                        ctxs[i].handle, C.c_void_p(gr["gh"].data_ptr()),
                        C.c_void_p(gr["mh"].data_ptr()) if gr["mh"] is not None else None,
                        gr["descs"], len(gr["descs"]), C.byref(opts[i]), C.byref(bv))
                    NN.check(rc)
                    d2h_box[i] += 52 * gr["n"] + 65 * int(bv.n_faces) + 4 * int(bv.n_connections)
            except Exception as e:  # re-raised on the main thread
                errors.append(e)

        def e2e_step():
            for i in range(nctx):
                d2h_box[i] = 0
            ts = [threading.Thread(target=worker, args=(i,)) for i in range(nctx)]
            for t in ts:
                t.start()
            for t in ts:
                t.join()
            if errors:
                raise errors[0]
            return sum(d2h_box)

        for _ in range(args.warmup):
            e2e_step()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(streams[0])
        for s_ in streams[1:]:
            s_.wait_event(e0)
        for _ in range(args.steps):
            d2h = e2e_step()
        for s_ in streams[1:]:
            streams[0].wait_stream(s_)
        e1.record(streams[0])
        torch.cuda.synchronize(dev)
        e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, dist, dev)
        for c in ctxs[1:]:
            c.close()
        h2d = sum(24 * gr["n"] + (gr["n"] if gr["mh"] is not None else 0) for gr in groups)
        e2e = {"value": aggregate_cells_per_s(world, n, e_ms), "unit": "cells/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e_ms,
               "contexts": nctx,
               "api": "mv_context_build_batch (host buffers), one context per host thread"}

    peak, peak_kind = measured_peaks()
    cells_ms = sum(st["ms_cells"] for st in stats)
    alg_bytes = BYTES_GEN * n + BYTES_CELL * n + BYTES_FACE * F + BYTES_CONN * Cn
    achieved = alg_bytes / (cells_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind,
                "kernel": "all cell kernels of the batch builds",
                "alg_bytes_per_launch": alg_bytes, "kernel_ms_per_launch": cells_ms}
    cb = None
    if rank == 0 and not args.no_cpu_baseline:
        cb = cpu_baseline_batch(jobs, budget_s=args.cpu_budget)
    if rank == 0:
        tot = lambda k: int(sum(st[k] for st in stats))
        line = {"metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic",
                "config": {"workload": f"batch_{njobs}_uneven_tessellations", "n_jobs": njobs,
                           "n_generators": n, "batch_builds_per_step": len(groups),
                           "precision": args.precision, "parallelism": f"weak{world}",
                           "cache": "inputs larger than L2"},
                "roofline": roofline, "cpu_baseline": cb, "e2e": e2e,
                "gpu_launches": tot("kernel_launches") * args.steps, "clocks": clocks,
                "phases_ms": {"grid": sum(st["ms_grid"] for st in stats), "cells": cells_ms,
                              "finalize": sum(st["ms_finalize"] for st in stats)},
                "counts": {"faces": F, "connections": Cn, "cells_built": tot("cells_built"),
                           "staged_wide": tot("staged_wide"), "staged_retries": tot("staged_retries"),
                           "overflow_cells": tot("overflow_cells")},
                "parity": parity}
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return HBM_PEAK_FALLBACK, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(w, budget_s=12.0, threads=None):
    """The oracle (C++ restatement of the reference algorithm) with OpenMP on all host
    cores on a bounded sample of the workload: the first m cells (spatially random for
    the Poisson workloads) as one partial build, m sized for about budget_s seconds of
    cell work.  value = m / the measured time of the sample's per-cell loop; the build's
    fixed costs (setup with the serial grid build, flatten) are reported beside it."""
    from oracle import oracle as O
    g, n = w["generators"], len(w["generators"])
    threads = threads or os.cpu_count()
    kw = dict(dim=w["dimensionality"], periodic=w["periodic"], nthreads=threads,
              flags=O.NO_CSR)

    def run(m):
        mask = np.zeros(n, dtype=bool)
        mask[:m] = True
        r = O.build(g, w["anchor"], w["width"], mask=mask, **kw)
        assert r.status == 0
        return r.times

    m = min(n, 100000)
    rate = m / max(run(m)[1], 1e-3)
    m = int(min(n, max(m, rate * budget_s)))
    t_setup, t_cells, t_fin = run(m)
    return {"value": m / t_cells, "unit": "cells/s", "cores": threads, "kind": "port",
            "sample": f"first {m} of the {n} cells of the same workload as one partial build: "
                      f"{t_cells:.1f} s of cell work measured (fixed costs of a build: "
                      f"{t_setup:.1f} s setup with the serial grid build, {t_fin:.1f} s flatten)"}


def reference_partition(w, steps, warmup, threads=None):
    """The reference arm on a single tessellation: the oracle on all host cores.  Step k
    builds the cells [k n / K, (k + 1) n / K) as one partial build, so the K steps
    together build every cell of the workload exactly once; the full build's time is
    one setup (generators, boundary, serial grid build) + the K steps' measured per-cell
    loops + one flatten, all measured (no extrapolation)."""
    from oracle import oracle as O
    g, n = w["generators"], len(w["generators"])
    threads = threads or os.cpu_count()
    kw = dict(dim=w["dimensionality"], periodic=w["periodic"], nthreads=threads,
              flags=O.NO_CSR)

    def run(a, b):
        mask = np.zeros(n, dtype=bool)
        mask[a:b] = True
        t0 = time.perf_counter()
        r = O.build(g, w["anchor"], w["width"], mask=mask, **kw)
        wall = time.perf_counter() - t0
        assert r.status == 0
        return wall, r.times

    for k in range(warmup):
        run(k * 1000, k * 1000 + min(n, 20000))
    K = max(1, steps)
    walls, setups, cells, fins = [], [], [], []
    for k in range(K):
        wall, (ts, tc, tf) = run(k * n // K, (k + 1) * n // K)
        walls.append(wall)
        setups.append(ts)
        cells.append(tc)
        fins.append(tf)
    full_s = float(np.median(setups)) + float(np.sum(cells)) + float(np.median(fins))
    return {"value": n / full_s, "ms_per_step": 1e3 * float(np.mean(walls)),
            "cpu_baseline": {
                "value": n / full_s, "unit": "cells/s", "cores": threads, "kind": "port",
                "full_build_s": full_s, "cell_loop_s": float(np.sum(cells)),
                "setup_s": float(np.median(setups)), "flatten_s": float(np.median(fins)),
                "sample": f"all {n} cells, each built once across the {K} steps (step k: the "
                          f"cells [k n/{K}, (k+1) n/{K}) as a partial build); full build = one "
                          f"setup + the steps' cell loops + one flatten, measured"}}


def reference_batch(jobs, steps, warmup, threads=None):
    """The reference arm on the batch: one oracle build per tessellation (as a caller of
    the reference loops over Voronoi::build); step k builds the k-th of K consecutive
    slices of the tessellations, so the K steps build every tessellation once."""
    from oracle import oracle as O
    threads = threads or os.cpu_count()

    def build(j):
        t0 = time.perf_counter()
        r = O.build(j["generators"], j["anchor"], j["width"], dim=j["dimensionality"],
                    periodic=j["periodic"], mask=j.get("mask"), nthreads=threads, flags=O.NO_CSR)
        assert r.status == 0
        return time.perf_counter() - t0

    for j in jobs[:warmup]:
        build(j)
    K = max(1, steps)
    nj = len(jobs)
    walls = []
    for k in range(K):
        walls.append(sum(build(j) for j in jobs[k * nj // K:(k + 1) * nj // K]))
    n = sum(len(j["generators"]) for j in jobs)
    total = float(np.sum(walls))
    return {"value": n / total, "ms_per_step": 1e3 * total / K,
            "cpu_baseline": {"value": n / total, "unit": "cells/s", "cores": threads,
                             "kind": "port", "full_build_s": total,
                             "sample": f"all {nj} tessellations ({n} cells), each built once "
                                       f"across the {K} steps, one build per tessellation"}}


def parity_single(w, dv, frac=0.01, seed=11):
    """Parity of the timed build (its device result dv, before anything else runs on the
    context) against the oracle, outside the timed region: workloads of at most
    FULL_PARITY_CELLS cells are compared in full, larger ones on a seeded sample of
    cells (the oracle's partial build of those cells, every face of each, against the
    faces the full GPU build gives them); the volume closure covers all cells."""
    from oracle import parity
    from meshless_voro_b200.voronoi import device_tensors
    n = len(w["generators"])
    t = device_tensors(dv)
    full = n <= FULL_PARITY_CELLS
    idx = np.arange(n) if full else parity.sample_cells(n, frac, seed)
    g = parity.device_sample(t, idx)
    o = parity.oracle_sample(w, idx, nthreads=os.cpu_count())
    res = parity.compare_sample(g, o)
    res["kind"] = "full" if full else f"sampled ({100 * len(idx) / n:.2f} % of the cells, seed {seed})"
    res["oracle_s"] = o["oracle_s"]
    res["closure"] = parity.closure(t["cell_volume"].cpu().numpy(), w["width"], w["dimensionality"])
    return res


def parity_batch(ctx, groups, jobs_by_group, per_group=2, seed=11, **build_kw):
    """Parity of batch builds: each batch build of the step runs again (untimed) and a
    seeded sample of its tessellations is compared in full with the oracle's builds of
    them alone (cells, faces in order, CSR, every value)."""
    import torch
    from oracle import oracle as O
    from oracle import parity
    from meshless_voro_b200.voronoi import device_tensors
    rng = np.random.default_rng(seed)
    tot = {"tessellations_compared": 0, "cells_compared": 0, "faces_compared": 0,
           "topology_mismatched_tessellations": 0, "max_rel_err": {}, "bit_identical": True}
    for gr, jobs in zip(groups, jobs_by_group):
        d_mask = gr["md"].data_ptr() if gr["md"] is not None else 0
        bv = ctx.build_batch_device(gr["gd"].data_ptr(), d_mask, gr["descs"], **build_kw)
        t = device_tensors(bv)
        co, fo, no = bv.job_cell_offset, bv.job_face_offset, bv.job_connection_offset
        for k in sorted(rng.choice(len(jobs), size=min(per_group, len(jobs)), replace=False)):
            j = jobs[k]
            c0, c1, f0, f1 = co[k], co[k + 1], fo[k], fo[k + 1]
            n0, n1 = no[k], no[k + 1]
            r = O.build(j["generators"], j["anchor"], j["width"], dim=j["dimensionality"],
                        periodic=j["periodic"], mask=j.get("mask"), nthreads=os.cpu_count())
            assert r.status == 0
            fl = t["face_left"][f0:f1].cpu().numpy()
            gv = {"volume": t["cell_volume"][c0:c1].cpu().numpy(),
                  "centroid": t["cell_centroid"][c0:c1].cpu().numpy(),
                  "safety_radius": t["cell_safety_radius"][c0:c1].cpu().numpy(),
                  "face_count": np.bincount(fl, minlength=c1 - c0), "face_left": fl,
                  "face_right": t["face_right"][f0:f1].cpu().numpy(),
                  "face_area": t["face_area"][f0:f1].cpu().numpy(),
                  "face_centroid": t["face_centroid"][f0:f1].cpu().numpy(),
                  "face_normal": t["face_normal"][f0:f1].cpu().numpy(),
                  "face_shift_code": t["face_shift_code"][f0:f1].cpu().numpy()}
            ov = {"volume": r.volume, "centroid": r.centroid, "safety_radius": r.safety_radius,
                  "face_count": np.bincount(r.face_left, minlength=c1 - c0),
                  "face_left": r.face_left, "face_right": r.face_right, "face_area": r.face_area,
                  "face_centroid": r.face_centroid, "face_normal": r.face_normal,
                  "face_shift_code": r.face_shift_code}
            res = parity.compare_sample(gv, ov)
            csr_ok = (np.array_equal(t["cell_face_offset"][c0:c1].cpu().numpy(), r.face_offset) and
                      np.array_equal(t["cell_face_connections"][n0:n1].cpu().numpy(),
                                     r.cell_face_connections))
            tot["tessellations_compared"] += 1
            tot["cells_compared"] += res["cells_compared"]
            tot["faces_compared"] += res["faces_compared"]
            if res["topology_mismatched_cells"] or not csr_ok:
                tot["topology_mismatched_tessellations"] += 1
            for key, v in res["max_rel_err"].items():
                tot["max_rel_err"][key] = max(tot["max_rel_err"].get(key, 0.0), v)
            tot["bit_identical"] = tot["bit_identical"] and res["bit_identical"] and csr_ok
        torch.cuda.synchronize()
    tot["rel_tol"] = parity.REL_TOL
    tot["ok"] = (tot["topology_mismatched_tessellations"] == 0 and
                 max(tot["max_rel_err"].values(), default=0.0) <= parity.REL_TOL)
    tot["kind"] = f"{per_group} tessellations per batch build, compared in full"
    return tot


def run_reference(args, rank, world):
    if rank != 0:
        return
    if args.workload.startswith("batch_"):
        from meshless_voro_b200 import workloads as W
        jobs = W.batch_jobs(njobs=int(args.workload.split("_")[1]), seed=rank_seed(0))
        res = reference_batch(jobs, args.steps, args.warmup)
        cfg = {"workload": f"batch_{len(jobs)}_uneven_tessellations",
               "n_jobs": len(jobs), "n_generators": sum(len(j["generators"]) for j in jobs),
               "precision": args.precision, "parallelism": f"weak{world}",
               "cache": "inputs larger than L2"}
    else:
        w = workload(args.workload, seed=rank_seed(0))
        res = reference_partition(w, args.steps, args.warmup)
        n = len(w["generators"])
        cfg = {"workload": w["name"], "n_generators": n,
               "periodic": w["periodic"], "precision": args.precision,
               "pipeline": args.pipeline, "parallelism": f"weak{world}",
               "cache": (f"inputs larger than L2 ({24 * n / 1e6:.0f} MB generators)"
                         if 24 * n >= L2_FLUSH_BYTES else
                         "L2 flushed (256 MB written) before each timed step")}
    v = res["value"]
    line = {"metric": METRIC, "value": v, "unit": "cells/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference", "config": cfg,
            "cpu_baseline": res["cpu_baseline"],
            "e2e": {"value": v, "unit": "cells/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": "the Rust reference cannot be built here (no cargo); the C++ restatement "
                    "of its algorithm (oracle/) runs on all host cores"}
    print(json.dumps(line), flush=True)


def e2e_single(args, w, g_host, ctx, dev, stream, dist, world, local):
    """End to end through the C ABI (mv_context_build): pinned host generators in, every
    result array copied back to pinned host memory, each step.  args.e2e_contexts
    contexts (the C ABI is thread-safe per context) run on as many host threads, each
    on its own stream, so one build's result copy overlaps another build's kernels; the
    steps are split between them and the whole is timed on the device (CUDA events: the
    first stream records the start and the others wait for it; the first stream waits
    for all of them before the end event)."""
    import ctypes as C
    import torch
    import meshless_voro_b200 as mv
    from meshless_voro_b200 import _native as NN
    nctx = max(1, min(args.e2e_contexts, args.steps))
    ctxs = [ctx] + [mv.Context(local) for _ in range(nctx - 1)]
    streams = [stream] + [torch.cuda.Stream(dev) for _ in range(nctx - 1)]
    opts = [mv.voronoi.make_options(args.precision, stream=s.cuda_stream) for s in streams]
    n = len(w["generators"])
    a3 = (C.c_double * 3)(*w["anchor"])
    w3 = (C.c_double * 3)(*w["width"])
    hv = [C.POINTER(NN.HostVoronoi)() for _ in ctxs]
    errors = []

    def run(i, count):
        try:
            for _ in range(count):
                rc = NN.lib().mv_context_build(ctxs[i].handle, C.c_void_p(g_host.data_ptr()), None,
                                               n, a3, w3, w["dimensionality"], int(w["periodic"]),
                                               C.byref(opts[i]), C.byref(hv[i]))
                NN.check(rc)
        except Exception as e:  # re-raised on the main thread
            errors.append(e)

    def all_threads(counts):
        ts = [threading.Thread(target=run, args=(i, c)) for i, c in enumerate(counts)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        if errors:
            raise errors[0]

    # warm-up: every context builds (sizes its workspace and pinned arena)
    all_threads([max(1, args.warmup // nctx)] * nctx)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(streams[0])
    for s in streams[1:]:
        s.wait_event(e0)
    counts = [args.steps // nctx + (1 if i < args.steps % nctx else 0) for i in range(nctx)]
    all_threads(counts)
    for s in streams[1:]:
        streams[0].wait_stream(s)
    e1.record(streams[0])
    torch.cuda.synchronize(dev)
    e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, dist, dev)
    h = hv[0].contents
    d2h = (8 + 24 + 8 + 8 + 4) * n + (4 + 4 + 8 + 24 + 24 + 1) * int(h.n_faces) + 4 * int(h.n_connections)
    for c in ctxs[1:]:
        c.close()
    return {"value": aggregate_cells_per_s(world, n, e_ms), "unit": "cells/s",
            "h2d_bytes_per_step": 24 * n, "d2h_bytes_per_step": d2h, "ms_per_step": e_ms,
            "contexts": nctx,
            "api": "mv_context_build (host buffers), one context per host thread"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="poisson_256")
    ap.add_argument("--precision", default="filtered", choices=["filtered", "fp64"])
    ap.add_argument("--pipeline", default="auto", choices=["auto", "staged", "fused"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-compare", action="store_true", help="skip the plain-FP64 side run")
    ap.add_argument("--e2e-contexts", type=int, default=2,
                    help="contexts (one host thread each) the end-to-end leg splits its steps over")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the (untimed) oracle comparison of the timed build")
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload.startswith("batch_"):
        run_batch(args, rank, world)
        return

    import torch
    import torch.distributed as dist
    import meshless_voro_b200 as mv

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", device_id=dev,
                                timeout=__import__("datetime").timedelta(seconds=120))

    w = workload(args.workload, seed=rank_seed(rank))
    n = len(w["generators"])
    g_host = torch.from_numpy(np.ascontiguousarray(w["generators"])).pin_memory()
    g_dev = g_host.to(dev)
    ctx = mv.Context(local)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream

    def step(precision, pipeline):
        return ctx.build_device(g_dev.data_ptr(), 0, n, w["anchor"], w["width"],
                                w["dimensionality"], w["periodic"], precision=precision,
                                stream=sp, pipeline=pipeline)

    # inputs smaller than L2: flush it (write a 256 MB buffer) before every timed step
    # and time each step alone
    flush = torch.empty(1 << 26, dtype=torch.float32, device=dev) if 24 * n < L2_FLUSH_BYTES else None

    def timed(precision, steps, pipeline=args.pipeline):
        for _ in range(args.warmup):
            step(precision, pipeline)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        per_step, stats, out = [], None, None
        if flush is None:
            e0.record(stream)
            for _ in range(steps):
                out = step(precision, pipeline)
                stats = ctx.last_stats()
                per_step.append(stats)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            ms_local = e0.elapsed_time(e1) / steps
        else:
            ms_local = 0.0
            for _ in range(steps):
                flush.fill_(1.0)
                e0.record(stream)
                out = step(precision, pipeline)
                e1.record(stream)
                torch.cuda.synchronize(dev)
                stats = ctx.last_stats()
                per_step.append(stats)
                ms_local += e0.elapsed_time(e1) / steps
        ms = max_over_ranks(ms_local, dist, dev)
        if world > 1:
            dist.barrier()
        # device times of the cell phase and its kernels (library CUDA events on `stream`)
        kms = {k: float(np.mean([st[k] for st in per_step]))
               for k in ("ms_cells", "ms_shell", "ms_clip", "ms_integrate", "ms_retry")}
        return ms, kms, stats, out

    with ClockSampler(local) as clk:
        ms, kms, stats, out = timed(args.precision, args.steps)
    clocks = clk.summary()
    F, Cn = int(out.n_faces), int(out.n_connections)
    # parity of the timed build against the oracle (untimed; before the context's next build)
    parity = None
    if rank == 0 and not args.no_parity:
        parity = parity_single(w, out)
    value = aggregate_cells_per_s(world, n, ms)
    cells_ms = kms["ms_cells"]

    # side by side: the other precision on the same pipeline, and the plain FP64 build
    # (the fused one-kernel-per-cell kernel, f64 predicates throughout)
    other = None
    if not args.no_compare:
        other = []
        o_prec = "fp64" if args.precision == "filtered" else "filtered"
        for prec, pipe, label in ((o_prec, args.pipeline, f"{o_prec}, same pipeline"),
                                  ("fp64", "fused", "plain FP64 per-cell kernel (fused)")):
            o_ms, o_kms, o_stats, _ = timed(prec, max(2, args.steps // 2), pipe)
            other.append({"label": label, "precision": prec, "pipeline": pipe,
                          "value": aggregate_cells_per_s(world, n, o_ms), "ms_per_step": o_ms,
                          "cells_ms": o_kms["ms_cells"],
                          "f32_undecided": o_stats["f32_undecided"],
                          "exact_tests": o_stats["exact_tests"]})

    # end to end through the C ABI with host buffers (pinned input, results to pinned host)
    e2e = None
    if not args.no_e2e:
        e2e = e2e_single(args, w, g_host, ctx, dev, stream, dist, world, local)

    peak, peak_kind = measured_peaks()
    # algorithmic bytes of the whole path for this workload (generator read, cell and
    # face outputs, CSR), counted from the run's own output
    alg_bytes = BYTES_GEN * n + BYTES_CELL * n + BYTES_FACE * F + BYTES_CONN * Cn
    staged = kms["ms_clip"] > 0.0
    if staged:
        # dominant kernel: the clip kernel; one launch per chunk of cells
        chunk = min(n, CHUNK_CELLS)
        launches = -(-n // chunk)
        per_launch_ms = kms["ms_clip"] / launches
        per_launch_bytes = alg_bytes * chunk / n
        traffic = (CLIP_KERNEL_DRAM_BYTES_PER_CELL * chunk
                   if args.workload.startswith("poisson") else None)
        kernel = "mv::clip_kernel (staged pipeline)"
    else:
        per_launch_ms, per_launch_bytes, traffic = cells_ms, alg_bytes, None
        kernel = "mv::cells_kernel (fused pipeline)"
    achieved = per_launch_bytes / (per_launch_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                "kernel": kernel, "alg_bytes_per_launch": per_launch_bytes,
                "kernel_ms_per_launch": per_launch_ms,
                "phase": {"kernels": "cell construction (all cell kernels)",
                          "achieved": alg_bytes / (cells_ms * 1e-3) / 1e9, "ms": cells_ms},
                "kernels_ms": {"shell": kms["ms_shell"], "clip": kms["ms_clip"],
                               "integrate": kms["ms_integrate"], "retry": kms["ms_retry"]}}

    cb = None
    if rank == 0 and not args.no_cpu_baseline:
        cb = cpu_baseline(workload(args.workload, seed=3), budget_s=args.cpu_budget)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic",
                "config": {"workload": w["name"], "n_generators": n, "periodic": w["periodic"],
                           "precision": args.precision, "pipeline": args.pipeline,
                           "parallelism": f"weak{world}",
                           "cache": (f"inputs larger than L2 ({24 * n / 1e6:.0f} MB generators)"
                                     if flush is None else
                                     "L2 flushed (256 MB written) before each timed step")},
                "roofline": roofline, "cpu_baseline": cb, "e2e": e2e,
                "gpu_launches": int(stats["kernel_launches"]) * args.steps,
                "clocks": clocks,
                "phases_ms": {"grid": stats["ms_grid"], "cells": stats["ms_cells"],
                              "finalize": stats["ms_finalize"]},
                "counts": {"faces": F, "connections": Cn,
                           "neighbours_clipped": stats["neighbours_clipped"],
                           "planes_added": stats["planes_added"],
                           "f32_undecided": stats["f32_undecided"],
                           "exact_tests": stats["exact_tests"],
                           "extra_shells": stats["extra_shells"],
                           "overflow_cells": stats["overflow_cells"],
                           "serial_rings": stats["serial_rings"],
                           "staged_retries": stats["staged_retries"]},
                "side_by_side": other, "parity": parity,
                "precision_comparison": None if not other else {
                    "filtered_vs_fp64_same_pipeline": (value / other[0]["value"]
                                                       if args.precision == "filtered"
                                                       else other[0]["value"] / value),
                    "default_vs_plain_fp64_fused_kernel": value / other[1]["value"]}}
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
