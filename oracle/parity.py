"""Parity of a GPU build against the oracle at full configuration sizes (TEST
INFRASTRUCTURE ONLY: the checker used by ``tests/`` and by ``bench.py`` outside its
timed region; the product library never imports it).

A full oracle build of the large configurations takes about a minute, so the large
ones are checked on a seeded random sample of their cells, the way the reference's
own partial-build test checks single cells against the full build
(voronoi.rs:1052-1085): the oracle builds only the sampled cells (a partial build,
every face of every built cell), and each sampled cell of the GPU's *full* build must
carry the same volume, centroid and safety radius, and exactly the faces the full
build assigns it -- the owned faces of voronoi_cell.rs:53-73 (boundary, periodic, or
towards a higher index), in the same clipping-plane order, with the same right cell,
shift, area, centroid and normal.  Every face of a tessellation is owned by exactly
one cell, so a uniform sample of cells is a uniform sample of faces.  The volume
closure of the reference's consistency check (voronoi.rs:398-406: the cell volumes
sum to the box volume) is evaluated over all cells with an exactly rounded sum.
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import oracle as O

REL_TOL = 1e-12  # integrals within 1e-12 relative of the oracle; topology bit-exact
CLOSURE_TOL = 1e-12


def sample_cells(n: int, frac: float, seed: int, min_cells: int = 1000) -> np.ndarray:
    """Sorted indices of a seeded uniform sample of max(frac * n, min_cells) cells."""
    m = int(min(n, max(min_cells, round(frac * n))))
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(n, size=m, replace=False))


def device_sample(t: dict, idx: np.ndarray) -> dict:
    """The sampled cells of a device result (torch views, see device_tensors): cell
    values, and the faces whose left cell is sampled, in face order (host numpy)."""
    import torch
    dev = t["cell_volume"].device
    ii = torch.as_tensor(idx, dtype=torch.int64, device=dev)
    out = {"volume": t["cell_volume"][ii].cpu().numpy(),
           "centroid": t["cell_centroid"][ii].cpu().numpy(),
           "safety_radius": t["cell_safety_radius"][ii].cpu().numpy()}
    fl = t["face_left"]
    lo = torch.searchsorted(fl, ii.to(torch.int32))
    hi = torch.searchsorted(fl, (ii + 1).to(torch.int32))
    cnt = hi - lo
    total = int(cnt.sum().item())
    start = torch.repeat_interleave(lo, cnt)
    first = torch.repeat_interleave(torch.cumsum(cnt, 0) - cnt, cnt)
    rows = start + (torch.arange(total, device=dev) - first)
    out["face_count"] = cnt.cpu().numpy()
    for k in ("face_left", "face_right", "face_area", "face_centroid", "face_normal",
              "face_shift_code"):
        out[k] = t[k][rows].cpu().numpy()
    return out


def host_sample(v, idx: np.ndarray) -> dict:
    """The same selection from a host result (VoronoiArrays-like)."""
    fl = np.asarray(v.face_left)
    lo = np.searchsorted(fl, idx, side="left")
    hi = np.searchsorted(fl, idx + 1, side="left")
    cnt = hi - lo
    rows = (np.concatenate([np.arange(a, b) for a, b in zip(lo, hi)]) if len(idx)
            else np.zeros(0, dtype=np.int64))
    return {"volume": v.cell_volume[idx], "centroid": v.cell_centroid[idx],
            "safety_radius": v.cell_safety_radius[idx], "face_count": cnt,
            "face_left": fl[rows], "face_right": v.face_right[rows], "face_area": v.face_area[rows],
            "face_centroid": v.face_centroid[rows], "face_normal": v.face_normal[rows],
            "face_shift_code": v.face_shift_code[rows]}


def oracle_sample(w: dict, idx: np.ndarray, nthreads: int = 0) -> dict:
    """The oracle's partial build of the sampled cells, every face of each, filtered to
    the faces the full build gives the cell (voronoi_cell.rs:53-73 without a mask)."""
    g = w["generators"]
    n = len(g)
    mask = np.zeros(n, dtype=bool)
    mask[idx] = True
    t0 = time.perf_counter()
    r = O.build(g, w["anchor"], w["width"], dim=w["dimensionality"], periodic=w["periodic"],
                mask=mask, nthreads=nthreads, flags=O.FACES_ALL | O.NO_CSR)
    secs = time.perf_counter() - t0
    if r.status != 0:
        raise RuntimeError(f"oracle build failed: status {r.status}, cell {r.error_cell}")
    owned = (r.face_right < 0) | (r.face_shift_code != 13) | (r.face_right > r.face_left)
    fl = r.face_left[owned]
    return {"volume": r.volume[idx], "centroid": r.centroid[idx],
            "safety_radius": r.safety_radius[idx],
            "face_count": np.bincount(np.searchsorted(idx, fl), minlength=len(idx)),
            "face_left": fl, "face_right": r.face_right[owned], "face_area": r.face_area[owned],
            "face_centroid": r.face_centroid[owned], "face_normal": r.face_normal[owned],
            "face_shift_code": r.face_shift_code[owned], "oracle_s": secs}


def _rel(a, b, scale):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.size == 0:
        return 0.0
    return float(np.max(np.abs(a - b) / (np.abs(b) + scale)))


def compare_sample(g: dict, o: dict) -> dict:
    """Topology (per-cell face counts, left / right / shift of every face, in order) must
    be identical; the integrals are compared relative to the oracle's (cell centroids
    and face centroids relative to the cells' length scale, as the GPU parity tests do)."""
    ncell = len(o["volume"])
    res = {"cells_compared": int(ncell), "faces_compared": int(len(o["face_left"]))}
    gc, oc = np.asarray(g["face_count"]), np.asarray(o["face_count"])
    same_counts = np.array_equal(gc, oc)
    if not same_counts:
        topo_bad = int(np.sum(gc != oc)) if gc.shape == oc.shape else ncell
    else:
        diff = ((np.asarray(g["face_left"]) != o["face_left"]) |
                (np.asarray(g["face_right"]) != o["face_right"]) |
                (np.asarray(g["face_shift_code"]).astype(np.int64) != o["face_shift_code"]))
        topo_bad = int(len(np.unique(np.asarray(o["face_left"])[diff])))
    res["topology_mismatched_cells"] = topo_bad
    vscale = float(np.max(np.abs(o["volume"]))) if ncell else 1.0
    lscale = vscale ** (1.0 / 3.0) if vscale > 0 else 1.0
    err = {"volume": _rel(g["volume"], o["volume"], 1e-300),
           "centroid": _rel(g["centroid"], o["centroid"], lscale),
           "safety_radius": _rel(g["safety_radius"], o["safety_radius"], 1e-300)}
    bit = (np.array_equal(g["volume"], o["volume"]) and np.array_equal(g["centroid"], o["centroid"])
           and np.array_equal(g["safety_radius"], o["safety_radius"]))
    if same_counts and topo_bad == 0:
        ascale = float(np.max(np.abs(o["face_area"]))) if len(o["face_area"]) else 1.0
        err["face_area"] = _rel(g["face_area"], o["face_area"], ascale * 1e-6)
        err["face_centroid"] = _rel(g["face_centroid"], o["face_centroid"], lscale)
        err["face_normal"] = _rel(g["face_normal"], o["face_normal"], 1.0)
        bit = bit and all(np.array_equal(g[k], o[k])
                          for k in ("face_area", "face_centroid", "face_normal"))
    res["max_rel_err"] = err
    res["bit_identical"] = bool(bit and same_counts and topo_bad == 0)
    res["rel_tol"] = REL_TOL
    res["ok"] = bool(same_counts and topo_bad == 0 and max(err.values()) <= REL_TOL)
    return res


def closure(volume: np.ndarray, width, dim: int) -> dict:
    """Sum of all cell volumes (exactly rounded, math.fsum) against the box volume."""
    box = 1.0
    for i in range(dim):
        box *= float(width[i])
    s = math.fsum(np.asarray(volume, dtype=np.float64).tolist())
    rel = abs(s - box) / box
    return {"volume_sum": s, "box_volume": box, "rel_err": rel, "tol": CLOSURE_TOL,
            "ok": bool(rel <= CLOSURE_TOL)}
