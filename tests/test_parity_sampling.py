"""The sampled-parity checker (oracle/parity.py) on the CPU: a full oracle build seen
through the sampling must agree with the oracle's partial build of the sampled cells
bit for bit, and a planted difference in the full build must be caught."""
import types

import numpy as np

from meshless_voro_b200 import workloads as W
from oracle import parity


def _as_arrays(r):
    return types.SimpleNamespace(
        cell_volume=r.volume, cell_centroid=r.centroid, cell_safety_radius=r.safety_radius,
        face_left=r.face_left, face_right=r.face_right, face_area=r.face_area,
        face_centroid=r.face_centroid, face_normal=r.face_normal,
        face_shift_code=r.face_shift_code)


def _workloads():
    rng = np.random.default_rng(21)
    yield W.poisson(6000, seed=5, periodic=True)
    yield dict(generators=W.perturbed_grid([0, 0, 0], [1, 1, 1], 12, 0.0, None),
               anchor=np.zeros(3), width=np.ones(3), dimensionality=3, periodic=True)
    yield dict(generators=rng.uniform(0, 1, (3000, 3)) * [2.0, 1.0, 0.5],
               anchor=np.zeros(3), width=np.array([2.0, 1.0, 0.5]), dimensionality=3,
               periodic=False)
    yield W.clustered(8000, 20, seed=8)


def test_sample_of_full_build_matches_partial_build(oracle):
    for w in _workloads():
        full = oracle.build(w["generators"], w["anchor"], w["width"], dim=w["dimensionality"],
                            periodic=w["periodic"])
        assert full.status == 0
        idx = parity.sample_cells(len(w["generators"]), 0.05, seed=1, min_cells=100)
        res = parity.compare_sample(parity.host_sample(_as_arrays(full), idx),
                                    parity.oracle_sample(w, idx))
        assert res["ok"] and res["bit_identical"], res
        assert res["faces_compared"] > 0
        cl = parity.closure(full.volume, w["width"], w["dimensionality"])
        assert cl["ok"], cl


def test_planted_differences_are_caught(oracle):
    w = W.poisson(4000, seed=6, periodic=True)
    full = oracle.build(w["generators"], w["anchor"], w["width"], dim=3, periodic=True)
    idx = parity.sample_cells(len(w["generators"]), 0.1, seed=2, min_cells=100)
    o = parity.oracle_sample(w, idx)
    # an integral off by one ulp: within tolerance but not bit-identical
    a = _as_arrays(full)
    a.face_area = a.face_area.copy()
    f = int(np.searchsorted(a.face_left, idx[3]))
    a.face_area[f] = np.nextafter(a.face_area[f], 2.0)
    res = parity.compare_sample(parity.host_sample(a, idx), o)
    assert res["ok"] and not res["bit_identical"]
    # a wrong neighbour: a topology mismatch in exactly one cell
    b = _as_arrays(full)
    b.face_right = b.face_right.copy()
    b.face_right[f] = (b.face_right[f] + 1) % len(w["generators"])
    res = parity.compare_sample(parity.host_sample(b, idx), o)
    assert not res["ok"] and res["topology_mismatched_cells"] == 1
    # a volume off by 1e-9 relative: outside tolerance; closure off as well
    c = _as_arrays(full)
    c.cell_volume = c.cell_volume.copy()
    c.cell_volume[idx[5]] *= 1.0 + 1e-9
    res = parity.compare_sample(parity.host_sample(c, idx), o)
    assert not res["ok"] and res["max_rel_err"]["volume"] > 1e-10
    c.cell_volume[0] += 1e-9
    assert not parity.closure(c.cell_volume, w["width"], 3)["ok"]
