"""The HDF5 layout of Voronoi::write_to_hdf5 (voronoi.rs:432-491) built from a result's
arrays: dataset paths and types, and the 2D face end points (voronoi.rs:462-483).
Runs on CPU over the oracle's arrays (the layout is the same function of the arrays
whichever build produced them)."""
import numpy as np
import pytest

import meshless_voro_b200 as mv
from meshless_voro_b200 import workloads as W
from meshless_voro_b200.voronoi import VoronoiArrays


def _arrays(oracle, g, dim, periodic, mask=None):
    r = oracle.build(g, [0, 0, 0], [1, 1, 1], dim=dim, periodic=periodic, mask=mask)
    assert r.status == 0
    return VoronoiArrays(
        n_cells=len(r.volume), anchor=np.zeros(3), width=np.ones(3), dimensionality=dim,
        periodic=periodic, cell_volume=r.volume, cell_centroid=r.centroid, cell_loc=r.loc,
        cell_safety_radius=r.safety_radius, cell_face_offset=r.face_offset,
        cell_face_count=r.face_count, face_left=r.face_left, face_right=r.face_right,
        face_area=r.face_area, face_centroid=r.face_centroid, face_normal=r.face_normal,
        face_shift_code=r.face_shift_code, cell_face_connections=r.cell_face_connections)


def test_layout_3d(oracle):
    g = np.random.default_rng(3).uniform(size=(400, 3))
    a = _arrays(oracle, g, 3, True)
    d = mv.Voronoi(a).hdf5_datasets()
    assert sorted(d) == sorted(["Cells/Volume", "Cells/FaceConnectionsOffset", "Cells/FaceCount",
                                "Cells/Centroid", "Cells/Generator", "Faces/Area", "Faces/Centroid",
                                "Faces/Normal", "CellFaceConnections"])
    assert d["Cells/Volume"].dtype == np.float64 and d["Cells/Volume"].shape == (400,)
    assert d["Cells/FaceCount"].dtype == np.uint64 and d["CellFaceConnections"].dtype == np.uint64
    assert d["Cells/Centroid"].shape == (400, 3) and d["Faces/Normal"].shape == (len(a.face_area), 3)
    assert np.array_equal(d["Cells/Generator"], g)
    assert np.array_equal(d["CellFaceConnections"], a.cell_face_connections)


def test_layout_2d_face_end_points(oracle):
    rng = np.random.default_rng(4)
    g = W.perturbed_plane([0, 0, 0], [1, 1, 1], 12, 0.8, rng)
    mask = rng.uniform(size=len(g)) < 0.8
    a = _arrays(oracle, g, 2, False, mask)
    d = mv.Voronoi(a).hdf5_datasets()
    s, e, c, n, area = (d["Faces/Start"], d["Faces/End"], d["Faces/Centroid"], d["Faces/Normal"],
                        d["Faces/Area"])
    assert s.shape == e.shape == c.shape
    # the segment of each face: its length is the face's area (a length in 2D), its
    # midpoint the centroid, its direction normal x Z
    assert np.allclose(np.linalg.norm(e - s, axis=1), area, rtol=1e-12, atol=1e-15)
    assert np.allclose(0.5 * (s + e), c, rtol=0, atol=1e-15)
    assert np.allclose(np.einsum("ij,ij->i", e - s, n), 0.0, atol=1e-15)
    assert np.all(s[:, 2] == c[:, 2])
    # inactive cells of a partial build are VoronoiCell::default()
    assert np.all(d["Cells/Volume"][~mask] == 0.0) and np.all(d["Cells/Generator"][~mask] == 0.0)


def test_save_datasets_round_trip(oracle, tmp_path):
    g = W.perturbed_plane([0, 0, 0], [1, 1, 1], 6, 0.5, np.random.default_rng(5))
    v = mv.Voronoi(_arrays(oracle, g, 2, True))
    v.save_datasets(tmp_path / "voronoi.npz")
    back = np.load(tmp_path / "voronoi.npz")
    for k, x in v.hdf5_datasets().items():
        assert np.array_equal(back[k], x), k


def test_write_to_hdf5_needs_h5py(oracle, tmp_path):
    try:
        import h5py  # noqa: F401
        pytest.skip("h5py is installed")
    except ImportError:
        pass
    v = mv.Voronoi(_arrays(oracle, np.random.default_rng(6).uniform(size=(50, 3)), 3, False))
    with pytest.raises(RuntimeError, match="h5py"):
        v.write_to_hdf5(tmp_path / "voronoi.hdf5")


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [2, 3])
def test_layout_of_gpu_build_matches_oracle(gpu_ctx, oracle, dim):
    rng = np.random.default_rng(7)
    g = (W.perturbed_plane([0, 0, 0], [1, 1, 1], 20, 0.9, rng) if dim == 2
         else rng.uniform(size=(2000, 3)))
    gpu = gpu_ctx.build_arrays(g, None, [0, 0, 0], [1, 1, 1], dim, True)
    dg = mv.Voronoi(gpu).hdf5_datasets()
    do = mv.Voronoi(_arrays(oracle, g, dim, True)).hdf5_datasets()
    assert sorted(dg) == sorted(do)
    for k in do:
        assert dg[k].dtype == do[k].dtype and np.array_equal(dg[k], do[k]), k
