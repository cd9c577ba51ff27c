"""Autotuner of the library's launch parameters, measured on a B200.

The reference builds every cell the same way on the host (voronoi.rs:265-315); on the
GPU the fastest way to build a tessellation depends on its dimensionality and size.
For each dimensionality and a ladder of build sizes this tuner times device-resident
builds of seeded uniform generator sets and picks, by coordinate descent, the
pipeline (fused one-kernel-per-cell or staged shell / clip / integral kernels), the
first neighbour shell's radius in mean spacings (how many neighbours are set up
first), the uniform grid's resolution (generators per grid cell) and the staged
pipeline's chunk.  The bands between measured sizes meet at geometric midpoints.

The table is written as JSON (``tuning/b200.json``) and as the library's built-in
header (``csrc/mv_tuning_table.h``, taken in at the next library build); at run time
``load_table`` installs a JSON table through ``mv_tuning_set``.  Results never depend
on the parameters, only the build time does.

    python -m meshless_voro_b200.autotune [--quick] [--write]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import time

from . import _native as N

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE_JSON = os.path.join(HERE, "tuning", "b200.json")
TABLE_HEADER = os.path.join(HERE, "csrc", "mv_tuning_table.h")
N_INF = 1 << 62

PIPELINES = {"staged": N.MV_PIPELINE_STAGED, "fused": N.MV_PIPELINE_FUSED}
PIPELINE_NAMES = {v: k for k, v in PIPELINES.items()}

# the ladder of measured sizes and the candidate values of each parameter
SIZES = {3: [1 << 12, 1 << 14, 1 << 16, 1 << 18, 1 << 20, 1 << 22, 1 << 24],
         2: [1 << 12, 1 << 14, 1 << 16, 1 << 18, 1 << 20, 1 << 22]}
RADII = {3: [2.2, 2.5, 2.8, 3.1, 3.4], 2: [2.0, 2.4, 2.8, 3.2], 1: [2.2]}
PPC = [1.5, 2.2, 3.0, 4.0]
CHUNKS = [1 << 18, 1 << 19, 1 << 20, 1 << 21]
DEFAULT_RADIUS = {3: 2.8, 2: 2.4, 1: 2.2}
STAGED_MIN = 65536  # the library's fixed rule before tuning


def _entry(d: dict) -> N.TuningEntry:
    e = N.TuningEntry()
    e.dimensionality = int(d["dimensionality"])
    e.pipeline = PIPELINES[d["pipeline"]]
    e.n_min = int(d["n_min"])
    e.n_max = int(d["n_max"])
    e.initial_radius = float(d["initial_radius"])
    e.points_per_grid_cell = float(d["points_per_grid_cell"])
    e.chunk_cells = int(d["chunk_cells"])
    return e


def read_table(path: str = TABLE_JSON) -> list:
    with open(path) as f:
        return json.load(f)["entries"]


def load_table(path: str = TABLE_JSON) -> None:
    """Installs a JSON table for this process (mv_tuning_set)."""
    entries = read_table(path)
    arr = (N.TuningEntry * len(entries))(*[_entry(d) for d in entries])
    N.check(N.lib().mv_tuning_set(arr, len(entries)))


def reset_table() -> None:
    """Back to the library's built-in table."""
    N.check(N.lib().mv_tuning_set(None, 0))


def lookup(dimensionality: int, n: int) -> dict:
    """The entry a build of n generators uses (mv_tuning_lookup)."""
    e = N.TuningEntry()
    N.check(N.lib().mv_tuning_lookup(int(dimensionality), int(n), C.byref(e)))
    return {"dimensionality": e.dimensionality, "pipeline": PIPELINE_NAMES[e.pipeline],
            "n_min": e.n_min, "n_max": e.n_max, "initial_radius": e.initial_radius,
            "points_per_grid_cell": e.points_per_grid_cell, "chunk_cells": e.chunk_cells}


def bands(sizes: list) -> list:
    """[n_min, n_max) around each measured size: bands meet at geometric midpoints,
    the first starts at 0 and the last is open."""
    out = []
    for i, n in enumerate(sizes):
        lo = 0 if i == 0 else int(math.sqrt(sizes[i - 1] * n))
        hi = N_INF if i == len(sizes) - 1 else int(math.sqrt(n * sizes[i + 1]))
        out.append((lo, hi))
    return out


def header_text(entries: list, source: str = "meshless_voro_b200/tuning/b200.json") -> str:
    lines = [
        "// mv_tuning_table.h -- built-in launch tuning of libmvgpu (generated by",
        "// `python -m meshless_voro_b200.autotune --write`; edit the JSON it reads from, not this).",
        f"// Source: {source}",
        "#pragma once",
        "// {dimensionality, pipeline, n_min, n_max, initial_radius, points_per_grid_cell,"
        " chunk_cells, reserved}",
        "static const mv_tuning_entry kBuiltinTuning[] = {",
    ]
    for d in entries:
        pipe = "MV_PIPELINE_STAGED" if d["pipeline"] == "staged" else "MV_PIPELINE_FUSED"
        nmax = f"{int(d['n_max'])}LL" if int(d["n_max"]) > 2 ** 31 else str(int(d["n_max"]))
        lines.append(f"    {{{int(d['dimensionality'])}, {pipe}, {int(d['n_min'])}, {nmax}, "
                     f"{float(d['initial_radius'])!r}, {float(d['points_per_grid_cell'])!r}, "
                     f"{int(d['chunk_cells'])}, 0}},")
    lines.append("};")
    return "\n".join(lines) + "\n"


def default_entries() -> list:
    """The library's fixed rule before tuning (also the rule for 1-D builds)."""
    out = []
    for dim in (1, 2, 3):
        for lo, hi, pipe in ((0, STAGED_MIN, "fused"), (STAGED_MIN, N_INF, "staged")):
            out.append({"dimensionality": dim, "pipeline": pipe, "n_min": lo, "n_max": hi,
                        "initial_radius": DEFAULT_RADIUS[dim], "points_per_grid_cell": 2.2,
                        "chunk_cells": 1 << 20})
    return out


# ------------------------------------------------------------------ measuring --
class _Bench:
    """Device-resident builds of one seeded uniform set, timed with CUDA events."""

    def __init__(self, ctx, dim: int, n: int, seed: int = 17):
        import numpy as np
        import torch
        from . import workloads as W
        w = W.poisson(n, seed=seed, periodic=True, dim=dim)
        self.w, self.n, self.dim = w, n, dim
        self.ctx = ctx
        self.g = torch.from_numpy(np.ascontiguousarray(w["generators"])).cuda()
        self.stream = torch.cuda.current_stream()
        # inputs below L2: flush it before every timed build
        self.flush = (torch.empty(1 << 26, dtype=torch.float32, device="cuda")
                      if 24 * n < (256 << 20) else None)

    def time_ms(self, params: dict, reps: int) -> float:
        import torch
        kw = dict(pipeline=params["pipeline"], initial_radius=params["initial_radius"],
                  points_per_grid_cell=params["points_per_grid_cell"],
                  chunk_cells=params["chunk_cells"] if params["pipeline"] == "staged" else 0)

        def one():
            self.ctx.build_device(self.g.data_ptr(), 0, self.n, self.w["anchor"], self.w["width"],
                                  self.dim, True, stream=self.stream.cuda_stream, **kw)

        one()
        ts = []
        for _ in range(reps):
            if self.flush is not None:
                self.flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(self.stream)
            one()
            e1.record(self.stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        ts.sort()
        return ts[len(ts) // 2]


def tune_size(ctx, dim: int, n: int, reps: int, log=print) -> dict:
    """Coordinate descent over pipeline, radius, grid resolution and chunk for one size."""
    b = _Bench(ctx, dim, n)
    base = {"pipeline": "staged" if n >= STAGED_MIN else "fused",
            "initial_radius": DEFAULT_RADIUS[dim], "points_per_grid_cell": 2.2,
            "chunk_cells": 1 << 20}
    t_default = b.time_ms(base, reps)
    best, t_best = dict(base), t_default
    axes = [("pipeline", ["fused", "staged"]), ("initial_radius", RADII[dim]),
            ("points_per_grid_cell", PPC)]
    if n > CHUNKS[0]:
        axes.append(("chunk_cells", [c for c in CHUNKS if c < 2 * n]))
    for _ in range(2):  # two sweeps over the axes
        changed = False
        for key, values in axes:
            if key == "chunk_cells" and best["pipeline"] != "staged":
                continue
            for v in values:
                if v == best[key]:
                    continue
                cand = dict(best, **{key: v})
                t = b.time_ms(cand, reps)
                if t < t_best * 0.985:  # a change must be a clear gain
                    best, t_best, changed = cand, t, True
        if not changed:
            break
    log(f"dim {dim} n {n}: default {t_default:.3f} ms -> tuned {t_best:.3f} ms {best}", flush=True)
    return dict(best, default_ms=t_default, tuned_ms=t_best, n=n)


def tune(dims=(3, 2), reps: int = 5, quick: bool = False, log=print) -> list:
    import torch
    from .voronoi import Context
    torch.cuda.init()
    reset_table()
    ctx = Context(0)
    entries = []
    for dim in dims:
        sizes = SIZES[dim][1::2] if quick else SIZES[dim]
        for (lo, hi), n in zip(bands(sizes), sizes):
            r = tune_size(ctx, dim, n, reps, log)
            entries.append({"dimensionality": dim, "pipeline": r["pipeline"], "n_min": lo, "n_max": hi,
                            "initial_radius": r["initial_radius"],
                            "points_per_grid_cell": r["points_per_grid_cell"],
                            "chunk_cells": r["chunk_cells"],
                            "measured": {"n": n, "default_ms": round(r["default_ms"], 4),
                                         "tuned_ms": round(r["tuned_ms"], 4)}})
    ctx.close()
    # 1-D builds keep the fixed rule
    entries += [e for e in default_entries() if e["dimensionality"] == 1]
    return entries


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--quick", action="store_true", help="every other size of the ladder")
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--write", action="store_true", help="write the JSON table and the header")
    ap.add_argument("--out", default=TABLE_JSON)
    ap.add_argument("--header", default=TABLE_HEADER)
    args = ap.parse_args()
    t0 = time.time()
    entries = tune(reps=args.reps, quick=args.quick)
    doc = {"device": _device_name(), "generated_s": round(time.time() - t0, 1),
           "workload": "seeded i.i.d. uniform generators, periodic unit box, device-resident inputs",
           "entries": entries}
    text = json.dumps(doc, indent=1)
    print(text)
    if args.write:
        os.makedirs(os.path.dirname(args.out), exist_ok=True)
        with open(args.out, "w") as f:
            f.write(text + "\n")
        with open(args.header, "w") as f:
            f.write(header_text(entries))


def _device_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name(0)
    except Exception:
        return "unknown"


if __name__ == "__main__":
    main()
