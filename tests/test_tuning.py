"""The launch-tuning table (CPU only: the lookup runs in the library without a GPU).

The committed JSON table and the library's built-in header must be the same table;
every band of it must be what mv_tuning_lookup returns at its edges; mv_tuning_set
must reject invalid entries and install valid ones; the tuner's bands must cover all
sizes without gaps."""
import os

import pytest

from meshless_voro_b200 import _native as N
from meshless_voro_b200 import autotune as A


@pytest.fixture(scope="module")
def lib():
    from meshless_voro_b200 import build as B
    B.build()
    L = N.lib()
    yield L
    L.mv_tuning_set(None, 0)


def test_header_is_the_json_table():
    with open(A.TABLE_HEADER) as f:
        assert f.read() == A.header_text(A.read_table())


def test_lookup_matches_every_band(lib):
    A.reset_table()
    entries = A.read_table()
    assert lib.mv_tuning_count() == len(entries)
    for d in entries:
        for n in (d["n_min"], d["n_max"] - 1, (d["n_min"] + d["n_max"]) // 2):
            e = A.lookup(d["dimensionality"], n)
            for k in ("pipeline", "n_min", "n_max", "chunk_cells"):
                assert e[k] == d[k], (d, n, k)
            assert e["initial_radius"] == pytest.approx(d["initial_radius"], rel=0, abs=0)
            assert e["points_per_grid_cell"] == d["points_per_grid_cell"]
    # every size of every dimensionality has exactly one band
    for dim in (1, 2, 3):
        bands = sorted((d["n_min"], d["n_max"]) for d in entries if d["dimensionality"] == dim)
        assert bands[0][0] == 0 and bands[-1][1] >= 1 << 62
        assert all(a[1] == b[0] for a, b in zip(bands, bands[1:]))


def test_set_rejects_and_installs(lib):
    good = {"dimensionality": 3, "pipeline": "fused", "n_min": 0, "n_max": 1 << 62,
            "initial_radius": 3.1, "points_per_grid_cell": 3.0, "chunk_cells": 1 << 19}
    bad = dict(good, initial_radius=-1.0)
    arr = (N.TuningEntry * 2)(A._entry(good), A._entry(bad))
    before = lib.mv_tuning_count()
    assert lib.mv_tuning_set(arr, 2) == N.MV_ERR_ARG
    assert lib.mv_tuning_count() == before
    assert lib.mv_tuning_set(arr, 1) == N.MV_OK
    e = A.lookup(3, 12345)
    assert e["pipeline"] == "fused" and e["initial_radius"] == 3.1 and e["chunk_cells"] == 1 << 19
    # a dimensionality without an entry falls back to the library's fixed rule
    e2 = A.lookup(2, 100000)
    assert e2["pipeline"] == "staged" and e2["initial_radius"] == 2.4
    A.reset_table()
    assert lib.mv_tuning_count() == len(A.read_table())


def test_bands_cover_all_sizes():
    sizes = A.SIZES[3]
    b = A.bands(sizes)
    assert b[0][0] == 0 and b[-1][1] == A.N_INF
    for (lo, hi), n in zip(b, sizes):
        assert lo <= n < hi
    assert all(x[1] == y[0] for x, y in zip(b, b[1:]))


def test_json_path_in_package():
    assert os.path.exists(A.TABLE_JSON)
