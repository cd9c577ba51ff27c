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
# 64^3 periodic Poisson case (profiles/clip_kernel_poisson64.md); traffic grows in
# proportion to the cells, so a launch's traffic is this figure times its cells.
CLIP_KERNEL_DRAM_BYTES_PER_CELL = 2438.4
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
    groups = []
    for grp in batch_groups(jobs):
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

    e2e = None
    if not args.no_e2e:
        opts = mv.voronoi.make_options(args.precision, stream=sp)

        def e2e_step():
            d2h = 0
            for gr in groups:
                bv = NN.BatchVoronoi()
                rc = NN.lib().mv_context_build_batch(
                    ctx.handle, C.c_void_p(gr["gh"].data_ptr()),
                    C.c_void_p(gr["mh"].data_ptr()) if gr["mh"] is not None else None,
                    gr["descs"], len(gr["descs"]), C.byref(opts), C.byref(bv))
                NN.check(rc)
                d2h += 52 * gr["n"] + 65 * int(bv.n_faces) + 4 * int(bv.n_connections)
            return d2h

        e_ms, d2h = timed(e2e_step)
        h2d = sum(24 * gr["n"] + (gr["n"] if gr["mh"] is not None else 0) for gr in groups)
        e2e = {"value": aggregate_cells_per_s(world, n, e_ms), "unit": "cells/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e_ms}

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
                           "overflow_cells": tot("overflow_cells")}}
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
    cores on a prefix of the workload's cells (cell order is spatially random for the
    Poisson workloads), extrapolated to all cells."""
    from oracle import oracle as O
    g, n = w["generators"], len(w["generators"])
    threads = threads or os.cpu_count()
    kw = dict(dim=w["dimensionality"], periodic=w["periodic"], nthreads=threads,
              flags=O.NO_CSR)

    def run(m):
        mask = np.zeros(n, dtype=bool)
        mask[:m] = True
        t0 = time.perf_counter()
        r = O.build(g, w["anchor"], w["width"], mask=mask, **kw)
        assert r.status == 0
        return time.perf_counter() - t0

    t_fixed = min(run(0), run(0))        # grid build + flatten (serial), no cells
    m = min(n, 200000)
    rate = m / max(run(m) - t_fixed, 1e-3)
    m = int(min(n, max(m, rate * budget_s)))
    t_cells = max(run(m) - t_fixed, 1e-6)
    full = t_fixed + t_cells * n / m
    return {"value": n / full, "unit": "cells/s", "cores": threads, "kind": "port",
            "sample": f"first {m} of the {n} cells of the same workload "
                      f"({t_cells:.1f} s of cell work + {t_fixed:.1f} s serial grid build, "
                      f"extrapolated to all cells)"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    if args.workload.startswith("batch_"):
        from meshless_voro_b200 import workloads as W
        jobs = W.batch_jobs(njobs=int(args.workload.split("_")[1]), seed=rank_seed(0))
        for _ in range(args.warmup):
            cpu_baseline_batch(jobs[:4], budget_s=1.0)
        vals, cb = [], None
        for _ in range(args.steps):
            cb = cpu_baseline_batch(jobs, budget_s=args.cpu_budget)
            vals.append(cb["value"])
        v = float(np.median(vals))
        n = sum(len(j["generators"]) for j in jobs)
        print(json.dumps({"metric": METRIC, "value": v, "unit": "cells/s", "n_gpus": args.gpus,
                          "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * n / v,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                          "dtype": "f64", "data": "synthetic", "impl": "reference",
                          "config": {"workload": args.workload, "n_generators": n},
                          "cpu_baseline": {**cb, "value": v},
                          "e2e": {"value": v, "unit": "cells/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return
    w = workload(args.workload, seed=3)
    n = len(w["generators"])
    vals = []
    for _ in range(args.warmup):
        cpu_baseline(w, budget_s=2.0)
    cb = None
    for _ in range(args.steps):
        cb = cpu_baseline(w, budget_s=args.cpu_budget)
        vals.append(cb["value"])
    v = float(np.median(vals))
    line = {"metric": METRIC, "value": v, "unit": "cells/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * n / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": w["name"], "n_generators": n, "periodic": w["periodic"],
                       "cache": "inputs larger than L2"},
            "cpu_baseline": {**cb, "value": v},
            "e2e": {"value": v, "unit": "cells/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": "Rust reference cannot be built here (no cargo); the C++ restatement "
                    "of its algorithm (oracle/) runs on all host cores"}
    print(json.dumps(line), flush=True)


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
        from meshless_voro_b200 import _native as NN
        import ctypes as C
        opts = mv.voronoi.make_options(args.precision, stream=sp)
        a3 = (C.c_double * 3)(*w["anchor"])
        w3 = (C.c_double * 3)(*w["width"])
        hv = C.POINTER(NN.HostVoronoi)()

        def e2e_step():
            rc = NN.lib().mv_context_build(ctx.handle, C.c_void_p(g_host.data_ptr()), None, n,
                                           a3, w3, w["dimensionality"], int(w["periodic"]),
                                           C.byref(opts), C.byref(hv))
            NN.check(rc)
            return hv.contents

        for _ in range(max(1, args.warmup)):
            e2e_step()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            h = e2e_step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, dist, dev)
        d2h = (8 + 24 + 8 + 8 + 4) * n + (4 + 4 + 8 + 24 + 24 + 1) * int(h.n_faces) + 4 * int(h.n_connections)
        e2e = {"value": aggregate_cells_per_s(world, n, e_ms), "unit": "cells/s",
               "h2d_bytes_per_step": 24 * n, "d2h_bytes_per_step": d2h, "ms_per_step": e_ms}

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
                "side_by_side": other}
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
