"""GPU parity of the cell export (VoronoiIntegrator's cells, decomposition, with_faces)
and of custom integrals, against the CPU oracle.

The planes, vertices, tets and face lists are the reference's own quantities
(convex_cell.rs:16-60, 89-187, 461-543); they must be identical, bit for bit.
"""
import zlib

import numpy as np
import pytest

import meshless_voro_b200 as mv
from meshless_voro_b200 import workloads as W
from meshless_voro_b200._native import MV_CELLS_TETS, MV_CELLS_WITH_FACES, MvError

pytestmark = pytest.mark.gpu


def _case(name):
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    if name == "poisson3k_periodic":
        return dict(g=rng.uniform(0, 1, (3000, 3)), a=[0, 0, 0], w=[1, 1, 1], dim=3, per=True)
    if name == "grid12_w2":
        return dict(g=W.perturbed_grid([0, 0, 0], [2, 2, 2], 12, 0.95, rng), a=[0, 0, 0],
                    w=[2, 2, 2], dim=3, per=False)
    if name == "lattice6_periodic":
        return dict(g=W.perturbed_grid([0, 0, 0], [1, 1, 1], 6, 0.0, None), a=[0, 0, 0],
                    w=[1, 1, 1], dim=3, per=True)
    if name == "clustered8k_periodic":
        return dict(g=W.clustered(8000, 20, seed=21)["generators"], a=[0, 0, 0], w=[1, 1, 1],
                    dim=3, per=True)
    if name == "plane20_periodic_2d":
        return dict(g=W.perturbed_plane([0, 0, 0], [1, 1, 1], 20, 0.9, rng), a=[0, 0, 0],
                    w=[1, 1, 1], dim=2, per=True)
    raise KeyError(name)


def _oracle(oracle, c, mask, faces):
    flags = oracle.EXPORT_CELLS | oracle.EXPORT_TETS | (oracle.EXPORT_FACES | oracle.WITH_FACES if faces else 0)
    r = oracle.build(c["g"], c["a"], c["w"], dim=c["dim"], periodic=c["per"], mask=mask, flags=flags)
    assert r.status == 0
    return r


def _compare(ca, ex, faces):
    assert np.array_equal(ca.plane_offset, ex["pl_off"])
    assert np.array_equal(ca.plane_normal, ex["pl_n"])
    assert np.array_equal(ca.plane_point, ex["pl_p"])
    assert np.array_equal(ca.plane_right, ex["pl_right"])
    assert np.array_equal(ca.plane_shift_code, ex["pl_code"])
    assert np.array_equal(ca.vertex_offset, ex["vx_off"])
    assert np.array_equal(ca.vertex_loc, ex["vx_loc"])
    assert np.array_equal(ca.vertex_dual, ex["vx_dual"])
    assert np.array_equal(ca.tet_offset, ex["tet_off"])
    assert np.array_equal(ca.tet_vertices, ex["tet_v"])
    assert np.array_equal(ca.tet_plane, ex["tet_plane"])
    if faces:
        assert np.array_equal(ca.face_offset, ex["cf_off"])
        assert np.array_equal(ca.face_plane, ex["cf_plane"])
        assert np.array_equal(ca.face_vertex_offset, ex["fv_off"])
        assert np.array_equal(ca.face_vertices, ex["fv"])


@pytest.mark.parametrize("pipeline", ["fused", "staged"])
@pytest.mark.parametrize("faces", [False, True])
@pytest.mark.parametrize("name", ["poisson3k_periodic", "grid12_w2", "lattice6_periodic",
                                  "plane20_periodic_2d", "clustered8k_periodic"])
def test_cells_export_parity(gpu_ctx, oracle, name, faces, pipeline):
    c = _case(name)
    if faces and c["dim"] != 3:
        pytest.skip("with_faces is 3D only")
    flags = MV_CELLS_TETS | (MV_CELLS_WITH_FACES if faces else 0)
    va, ca = gpu_ctx.build_cells(c["g"], None, c["a"], c["w"], c["dim"], c["per"],
                                 cells_flags=flags, pipeline=pipeline)
    r = _oracle(oracle, c, None, faces)
    _compare(ca, r.cells_export, faces)
    assert np.array_equal(va.cell_volume, r.volume) or faces  # fan integrals round differently


def test_cells_export_partial(gpu_ctx, oracle):
    c = _case("grid12_w2")
    n = len(c["g"])
    mask = np.random.default_rng(5).uniform(size=n) < 0.3
    va, ca = gpu_ctx.build_cells(c["g"], mask, c["a"], c["w"], 3, False,
                                 cells_flags=MV_CELLS_TETS | MV_CELLS_WITH_FACES)
    r = _oracle(oracle, c, mask, True)
    _compare(ca, r.cells_export, True)
    assert np.all(np.diff(ca.vertex_offset)[~mask] == 0)


def test_with_faces_is_3d_only(gpu_ctx):
    c = _case("plane20_periodic_2d")
    with pytest.raises(MvError) as e:
        gpu_ctx.build_cells(c["g"], None, c["a"], c["w"], 2, True,
                            cells_flags=MV_CELLS_TETS | MV_CELLS_WITH_FACES)
    assert e.value.status == 1
    vi = mv.VoronoiIntegrator.build(c["g"], None, c["a"], c["w"], 2, True, context=gpu_ctx)
    with pytest.raises(ValueError):
        vi.with_faces()


class SecondMoment:
    """A custom CellIntegral: the second moment of the cell about its generator."""

    def __init__(self):
        self.m2 = 0.0

    @classmethod
    def init(cls, cell):
        return cls()

    def collect(self, v0, v1, v2, gen):
        vol = mv.voronoi.signed_volume_tet(tuple(v0), tuple(v1), tuple(v2), tuple(gen))
        d = [float(v0[i]) + float(v1[i]) + float(v2[i]) - 3.0 * float(gen[i]) for i in range(3)]
        self.m2 += vol * (d[0] * d[0] + d[1] * d[1] + d[2] * d[2])

    def finalize(self):
        return self


class ScaledArea:
    """A custom FaceIntegral with data: the face area times a per-cell factor."""

    def __init__(self, f):
        self.f, self.area = f, 0.0

    @classmethod
    def init_with_data(cls, cell, plane_idx, data):
        return cls(float(data))

    @classmethod
    def init(cls, cell, plane_idx):
        return cls(1.0)

    def collect(self, v0, v1, v2, gen):
        self.area += self.f * mv.voronoi.signed_area_tri(tuple(v0), tuple(v1), tuple(v2), tuple(gen))

    def finalize(self):
        return self


def _oracle_cell_integral(integral, r, k):
    ex = r.cells_export
    it = integral.init(None)
    for v in ex["tet_v"][ex["tet_off"][k]:ex["tet_off"][k + 1]]:
        it.collect(v[0], v[1], v[2], r.loc[k])
    return it.finalize()


@pytest.mark.parametrize("faces", [False, True])
def test_custom_integrals(gpu_ctx, oracle, faces):
    c = _case("poisson3k_periodic")
    vi = mv.VoronoiIntegrator.build(c["g"][:600], None, c["a"], c["w"], 3, True, context=gpu_ctx)
    if faces:
        vi = vi.with_faces()
    r = oracle.build(c["g"][:600], c["a"], c["w"], dim=3, periodic=True,
                     flags=oracle.EXPORT_TETS | (oracle.WITH_FACES if faces else 0))
    got = vi.compute_cell_integrals(SecondMoment)
    for k in range(0, 600, 37):
        assert got[k].m2 == _oracle_cell_integral(SecondMoment, r, k).m2
    # the built-in integrals through the crate's protocol: the fan decomposition's volumes
    # are the oracle's WITH_FACES volumes, bit for bit
    vols = vi.compute_cell_integrals(mv.VolumeCentroidIntegral)
    assert np.array_equal(np.array([v.volume for v in vols]), r.volume)
    # custom face integrals: non-symmetric = every valid face (FACES_ALL), symmetric = each
    # face once (the owned faces); areas bit-identical to the oracle's sums
    fl = oracle.WITH_FACES if faces else 0
    r_all = oracle.build(c["g"][:600], c["a"], c["w"], dim=3, periodic=True, flags=oracle.FACES_ALL | fl)
    r_own = oracle.build(c["g"][:600], c["a"], c["w"], dim=3, periodic=True, flags=fl)
    fa = vi.compute_face_integrals(ScaledArea)
    fs = vi.compute_face_integrals_sym(ScaledArea)
    assert np.array_equal(np.array([f.integral().area for f in fa]), r_all.face_area)
    assert np.array_equal(np.array([f.left() for f in fa]), r_all.face_left)
    assert np.array_equal(np.array([f.integral().area for f in fs]), r_own.face_area)
    # with per-cell data
    data = np.linspace(1.0, 2.0, 600)
    fd = vi.compute_face_integrals_sym_with_data(ScaledArea, data)
    assert [f.left() for f in fd] == [f.left() for f in fs]
    assert all(f.integral().f == data[f.left()] for f in fd)


def test_get_cell_at_with_faces(gpu_ctx, oracle):
    c = _case("grid12_w2")
    vi = mv.VoronoiIntegrator.build(c["g"], None, c["a"], c["w"], 3, False, context=gpu_ctx).with_faces()
    cell = vi.get_cell_at(100)
    r = _oracle(oracle, c, None, True)
    ex = r.cells_export
    f0, f1 = ex["cf_off"][100], ex["cf_off"][101]
    assert cell.face_count() == f1 - f0
    for f in range(cell.face_count()):
        k = ex["cf_plane"][f0 + f]
        s, e = ex["fv_off"][f0 + f], ex["fv_off"][f0 + f + 1]
        assert np.array_equal(cell.face_vertices(f), ex["fv"][s:e])
        assert cell.neighbour(f) == (None if ex["pl_right"][ex["pl_off"][100] + k] < 0
                                     else ex["pl_right"][ex["pl_off"][100] + k])
    assert len(list(vi.cells_iter())) == len(c["g"])
