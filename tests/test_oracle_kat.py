"""Pins the CPU oracle against the reference crate's own known-answer tests.

Each test cites the reference test it restates (meshless_voronoi 0.7.2).  The
reference's tests draw unseeded points (thread_rng); these use seeded PCG64 draws of
the same distributions.
"""
import json
import math
import os

import numpy as np
import pytest

from meshless_voro_b200.workloads import perturbed_grid, perturbed_plane
from voronoi_checks import approx_eq, consistency_check

HERE = os.path.dirname(os.path.abspath(__file__))


def test_single_cell(oracle):  # voronoi.rs:903-909
    r = oracle.build([[0.5, 0.5, 0.5]], [0, 0, 0], [1, 1, 1])
    assert r.status == 0
    assert approx_eq(r.volume[0], 1.0)


def test_two_cells(oracle):  # voronoi.rs:912-930
    r = oracle.build([[0.3, 0.4, 0.25], [0.7, 0.6, 0.75]], [0, 0, 0], [1, 1, 1])
    assert approx_eq(r.volume[0], 0.5) and approx_eq(r.volume[1], 0.5)


def test_4_cells(oracle):  # voronoi.rs:933-966
    g = [[0.4, 0.3, 0], [1.6, 0.2, 0], [0.6, 0.8, 0], [1.4, 0.7, 0]]
    r = oracle.build(g, [0, 0, 0], [2, 1, 1], dim=2, periodic=True)
    assert r.status == 0
    consistency_check(r, 2, [2, 1, 1])


def test_five_cells(oracle):  # voronoi.rs:969-1006
    d = math.sqrt(0.1)
    g = [[0.5, 0.5, 0.5], [0.5 - d, 0.5 - d, 0.5], [0.5 - d, 0.5 + d, 0.5],
         [0.5 + d, 0.5 + d, 0.5], [0.5 + d, 0.5 - d, 0.5]]
    r = oracle.build(g, [0, 0, 0], [1, 1, 1], dim=2)
    for v in r.volume:
        assert approx_eq(v, 0.2)


@pytest.mark.parametrize("n", [2, 3, 4])
def test_lattice_cells(oracle, n):  # voronoi.rs:1009-1039 (eight/27/64 cells)
    g = perturbed_grid([0, 0, 0], [1, 1, 1], n, 0.0, None)
    r = oracle.build(g, [0, 0, 0], [1, 1, 1])
    assert r.status == 0
    for v in r.volume:
        assert approx_eq(v, 1.0 / n ** 3)
    assert r.stats[:, 4].sum() > 0  # the exact predicate decided the co-spherical cases


def test_125_cells(oracle):  # voronoi.rs:1042-1049
    g = perturbed_grid([0, 0, 0], [1, 1, 1], 5, 0.5, np.random.default_rng(125))
    r = oracle.build(g, [0, 0, 0], [1, 1, 1])
    consistency_check(r, 3, [1, 1, 1])


def test_partial(oracle):  # voronoi.rs:1052-1085
    g = perturbed_grid([0, 0, 0], [1, 1, 1], 3, 0.9, np.random.default_rng(27))
    full = oracle.build(g, [0, 0, 0], [1, 1, 1])
    for i in range(27):
        mask = np.zeros(27, dtype=bool)
        mask[i] = True
        part = oracle.build(g, [0, 0, 0], [1, 1, 1], mask=mask)
        for j in range(27):
            if j == i:
                assert approx_eq(full.volume[j], part.volume[j])
                assert full.face_count[j] == part.face_count[j]
            else:
                assert part.volume[j] == 0.0


def test_2_d(oracle):  # voronoi.rs:1088-1110
    g = perturbed_plane([2, 2, 2], [2, 2, 1], 25, 0.95, np.random.default_rng(2))
    r = oracle.build(g, [2, 2, 2], [2, 2, 1], dim=2, periodic=True)
    assert approx_eq(r.volume.sum(), 4.0, epsilon=1e-10, ulps=8)


def test_3_d(oracle):  # voronoi.rs:1113-1122
    g = perturbed_grid([0, 0, 0], [2, 2, 2], 15, 0.95, np.random.default_rng(3))
    r = oracle.build(g, [0, 0, 0], [2, 2, 2])
    assert len(r.volume) == len(g)
    consistency_check(r, 3, [2, 2, 2])


def test_density_grad_2_d(oracle):  # voronoi.rs:1125-1155
    rng = np.random.default_rng(4)
    parts = []
    for i, count in enumerate([10, 40, 20, 80]):
        parts.append(perturbed_plane([0.25 * i, 0, 0], [0.25, 1, 1], count, 1.0, rng))
    g = np.concatenate(parts)
    r = oracle.build(g, [0, 0, 0], [1, 1, 1], dim=2, periodic=True)
    assert r.status == 0 and len(r.volume) == len(g)
    consistency_check(r, 2, [1, 1, 1])


def test_degenerate(oracle):  # voronoi.rs:1158-1165
    g = perturbed_grid([0, 0, 0], [2e15] * 3, 10, 0.0, None)
    g[42] = 1e14 * np.array([1.00007490802, 9.00019014286, 5.00014639879])
    r = oracle.build(g, [0, 0, 0], [2e15] * 3)
    assert r.status == 0
    consistency_check(r, 3, [2e15] * 3)


def test_degenerate_simplified(oracle):  # voronoi.rs:1168-1184
    anchor, width = [0.0, 6e14, 2e14], [6e14] * 3
    g = perturbed_grid(anchor, width, 3, 0.0, None)
    g[4] = 1e14 * np.array([1.00007490802, 9.00019014286, 5.00014639879])
    mask = np.zeros(27, dtype=bool)
    mask[3] = True
    r = oracle.build(g, anchor, width, mask=mask)
    assert r.status == 0
    consistency_check(r, 3, width)


def test_integrator_faces_match_voronoi(oracle):  # voronoi.rs:1187-1245
    g = perturbed_grid([0, 0, 0], [2, 2, 2], 5, 0.95, np.random.default_rng(5))
    mask = np.zeros(125, dtype=bool)
    mask[62] = True
    vor = oracle.build(g, [0, 0, 0], [2, 2, 2], periodic=True, mask=mask)
    allf = oracle.build(g, [0, 0, 0], [2, 2, 2], periodic=True, mask=mask,
                        flags=oracle.FACES_ALL)
    assert len(allf.face_area) == len(vor.face_area)
    assert np.array_equal(allf.face_area, vor.face_area)
    assert np.array_equal(allf.face_centroid, vor.face_centroid)
    assert vor.volume[62] == allf.volume[62]
    assert np.array_equal(vor.centroid[62], allf.centroid[62])


def test_non_perturbed_z(oracle):  # voronoi.rs:1248-1296 (fixture tests/golden)
    fx = json.load(open(os.path.join(HERE, "golden", "non_perturbed_z.json")))
    r = oracle.build(fx["generators"], fx["anchor"], fx["width"])
    assert r.status == 0
    consistency_check(r, 3, fx["width"])


def test_insphere_equivalence(oracle):  # geometry.rs:509-547
    rng = np.random.default_rng(10000)
    checked = 0
    for _ in range(10000):
        tet = rng.uniform(0, 1, size=(4, 3))
        v1, v2, v3 = tet[0] - tet[1], tet[0] - tet[2], tet[0] - tet[3]
        normal = np.cross(v1, v2)
        normal /= np.linalg.norm(normal)
        if normal @ v3 < 0:
            continue
        p1 = (v1 / np.linalg.norm(v1), tet[0] + 0.5 * v1)
        p2 = (v2 / np.linalg.norm(v2), tet[0] + 0.5 * v2)
        p3 = (v3 / np.linalg.norm(v3), tet[0] + 0.5 * v3)
        vert = oracle.intersect_planes(*p1, *p2, *p3)
        ngb = rng.uniform(0, 1, size=3)
        v4 = tet[0] - ngb
        clip_plane = oracle.half_space_clip(v4 / np.linalg.norm(v4), tet[0] + 0.5 * v4, vert)
        ilocs = [oracle.iloc([0, 0, 0], [1, 1, 1], p) for p in (*tet, ngb)]
        s_f64 = math.copysign(1.0, oracle.in_sphere_f64(*tet, ngb))
        s_exact = oracle.in_sphere_exact(*ilocs)
        assert clip_plane == s_f64
        assert clip_plane == s_exact
        checked += 1
    assert checked > 1000


def test_simple_cycle_extend(oracle):  # simple_cycle.rs:107-132
    tris = [(2, 4, 1), (1, 5, 2), (5, 1, 3), (5, 3, 6), (3, 4, 6), (4, 3, 1)]
    assert oracle.simple_cycle(tris, 7) == [2, 4, 6, 5]


def test_signed_volume(oracle):  # geometry.rs:368-379
    v0, v1, v2, v3 = [0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]
    vol = oracle.signed_volume_tet(v0, v1, v2, v3)
    assert vol == 1.0 / 6.0
    assert oracle.signed_volume_tet(v0, v2, v1, v3) == -vol


def test_signed_area(oracle):  # geometry.rs:381-402
    v0, v1, v2, t = [0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]
    a = oracle.signed_area_tri(v0, v1, v2, t)
    assert a == 0.5
    assert oracle.signed_area_tri(v0, v2, v1, t) == -a
    assert oracle.signed_area_tri(v0, v1, v2, [10, 10, 1]) == a


def test_clipping(oracle):  # convex_cell.rs:769-799
    assert oracle.clip_count([1, 1, 1], [2, 2, 2], [2, 2, 2], [2.5, 2.5, 2.5]) == 7


def test_extract_vertices(oracle):  # tests/test_extract_vertices.rs:41-152
    rng = np.random.default_rng(42)
    g = 3.0 * rng.uniform(0, 1, size=(1000, 3))
    a = oracle.build(g, [0, 0, 0], [3, 3, 3], flags=oracle.FACES_ALL)
    b = oracle.build(g, [0, 0, 0], [3, 3, 3], flags=oracle.FACES_ALL | oracle.WITH_FACES)
    assert np.allclose(a.volume, b.volume, rtol=0, atol=1e-10)
    assert np.array_equal(a.face_left, b.face_left)
    assert np.array_equal(a.face_right, b.face_right)
    assert np.allclose(a.face_area, b.face_area, rtol=0, atol=1e-10)
    assert np.allclose(a.centroid, b.centroid, rtol=0, atol=1e-5)
    assert np.allclose(a.face_centroid, b.face_centroid, rtol=0, atol=1e-5)
    assert np.array_equal(a.face_normal, b.face_normal)


@pytest.mark.parametrize("dim,periodic", [(3, False), (3, True), (2, True), (2, False), (1, True)])
def test_grid_stream_matches_brute_force(oracle, dim, periodic):
    rng = np.random.default_rng(dim * 10 + periodic)
    n = {3: 1500, 2: 800, 1: 60}[dim]
    g = rng.uniform(0, 1, size=(n, 3))
    a = oracle.build(g, [0, 0, 0], [1, 1, 1], dim=dim, periodic=periodic)
    b = oracle.build(g, [0, 0, 0], [1, 1, 1], dim=dim, periodic=periodic, flags=oracle.BRUTE_FORCE)
    assert a.status == 0 and b.status == 0
    for field in ("volume", "centroid", "safety_radius", "face_left", "face_right", "face_area",
                  "face_centroid", "face_normal", "face_shift_code", "cell_face_connections"):
        assert np.array_equal(getattr(a, field), getattr(b, field)), field


def test_duplicate_generators_error(oracle):  # convex_cell.rs:325-342 panics
    g = [[0.2, 0.2, 0.2], [0.7, 0.7, 0.7], [0.2, 0.2, 0.2]]
    r = oracle.build(g, [0, 0, 0], [1, 1, 1])
    assert r.status == 2


def test_box_corners_in_sphere_is_exactly_zero(oracle):
    """The exact predicate's shortcut: any five corners of one axis-aligned box (on
    each axis at most two of the iloc integers) have an exactly zero in-sphere
    determinant -- they lie on the box's circumsphere, or in one plane."""
    rng = np.random.default_rng(77)
    for _ in range(3000):
        lo = rng.integers(0, 1 << 51, size=3)
        hi = lo + rng.integers(0, 1 << 50, size=3) * rng.integers(0, 2, size=3)
        corners = [[(lo, hi)[(m >> i) & 1][i] for i in range(3)] for m in range(8)]
        pts = [corners[k] for k in rng.integers(0, 8, size=5)]
        assert oracle.in_sphere_exact(*pts) == 0.0
    # and a perturbed corner is (almost always) not
    nz = 0
    for _ in range(200):
        lo = rng.integers(0, 1 << 51, size=3)
        hi = lo + rng.integers(1, 1 << 50, size=3)
        corners = [[(lo, hi)[(m >> i) & 1][i] for i in range(3)] for m in range(8)]
        pts = [corners[k] for k in rng.permutation(8)[:5]]
        pts[4] = [pts[4][0] + 1, pts[4][1], pts[4][2]]
        nz += oracle.in_sphere_exact(*pts) != 0.0
    assert nz > 150
