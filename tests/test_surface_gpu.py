"""Device iso-surface (model.marching_cubes / extract_surface) against the CPU oracle:
identical vertices (FP32, every operation rounded alike) and faces on spheres, noise and
ragged shapes; closed, consistently oriented surfaces; the connectivity filter, Taubin
smoothing and the reference's errors; and the whole model path (reconstructed volume ->
Otsu threshold -> surface -> STL)."""
import numpy as np
import pytest
import torch

from oracle import model as om
from oracle import phantom as oph
from tomography_local_demo_b200 import SliceReconstructor, circular_cone_vectors
from tomography_local_demo_b200 import model as M

pytestmark = pytest.mark.gpu


def _closed_and_oriented(P, F):
    d = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
    und, cnt = np.unique(np.sort(d, axis=1), axis=0, return_counts=True)
    return bool(np.all(cnt == 2)) and len(np.unique(d, axis=0)) == len(d), len(P) - len(und) + len(F)


def _sphere(n, r, c=(0.0, 0.0, 0.0)):
    x = np.arange(n) - (n - 1) / 2
    X, Y, Z = np.meshgrid(x - c[0], x - c[1], x - c[2], indexing="ij")
    return (r - np.sqrt(X ** 2 + Y ** 2 + Z ** 2)).astype(np.float32)


def _cases():
    rng = np.random.default_rng(3)
    yield "sphere", _sphere(48, 15.0), 0.0, (-3.0, 1.0, 2.0), 0.25
    n = rng.normal(size=(37, 29, 41)).astype(np.float32)
    yield "noise", n, 0.2, (0.0, 0.0, 0.0), 1.0
    yield "noise-low-iso", n, -0.7, (1.0, 1.0, 1.0), 0.3
    yield "thin", rng.normal(size=(2, 9, 7)).astype(np.float32), 0.0, (0.0, 0.0, 0.0), 1.0
    yield "odd", rng.random((5, 130, 3)).astype(np.float32), 0.5, (0.0, -1.0, 0.0), 2.0


@pytest.mark.parametrize("name,vol,iso,origin,h", list(_cases()), ids=[c[0] for c in _cases()])
def test_marching_cubes_equals_oracle(cuda, name, vol, iso, origin, h):
    P, F = M.marching_cubes(torch.from_numpy(vol).cuda(), iso, origin, h)
    want_P, want_F = om.marching_cubes(vol, iso, origin, h)
    np.testing.assert_array_equal(P.cpu().numpy(), want_P)
    np.testing.assert_array_equal(F.cpu().numpy(), want_F)


@pytest.mark.parametrize("name,vol,iso,origin,h", list(_cases()), ids=[c[0] for c in _cases()])
def test_device_vertices_are_the_contour_edge_crossings(cuda, name, vol, iso, origin, h):
    """The device surface has exactly the vertex set that any marching-cubes contour of
    the reference (VTK flying edges or scikit-image) has: one vertex per crossed grid
    edge at the linear interpolation point (restated in test_surface.py from that
    definition alone), to FP32 rounding."""
    from test_surface import assert_same_vertex_set, edge_crossing_vertices
    P, _ = M.marching_cubes(torch.from_numpy(vol).cuda(), iso, origin, h)
    want = edge_crossing_vertices(vol, iso, origin, h)
    scale = max(1.0, float(np.abs(want).max()))
    assert_same_vertex_set(P.cpu().numpy(), want, 4e-6 * scale)


def test_sphere_surface_closed_with_the_right_area(cuda):
    P, F = M.marching_cubes(_sphere(96, 40.0), 0.0)
    P, F = P.cpu().numpy().astype(np.float64), F.cpu().numpy()
    ok, euler = _closed_and_oriented(P, F)
    assert ok and euler == 2
    tri = P[F]
    area = 0.5 * np.linalg.norm(np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0]), axis=1).sum()
    volume = np.einsum("ij,ij->i", tri[:, 0], np.cross(tri[:, 1], tri[:, 2])).sum() / 6
    assert abs(area / (4 * np.pi * 40.0 ** 2) - 1) < 0.005
    assert abs(volume / (4 / 3 * np.pi * 40.0 ** 3) - 1) < 0.005


def test_extract_surface_filter_smooth_errors(cuda, tmp_path):
    vol = np.maximum(_sphere(64, 20.0, (-8, 0, 0)), _sphere(64, 2.0, (22, 20, 20)))
    full = M.extract_surface(vol, (0, 0, 0), 1.0, 0.0, smooth=0, min_piece=0.0)
    big = M.extract_surface(vol, (0, 0, 0), 1.0, 0.0, smooth=0, min_piece=0.05)
    assert len(big["faces"]) < len(full["faces"])
    ok, euler = _closed_and_oriented(big["points"], big["faces"])
    assert ok and euler == 2                                  # the small sphere is gone
    sm = M.extract_surface(vol, (0, 0, 0), 1.0, 0.0, smooth=15, min_piece=0.05)
    assert np.array_equal(sm["faces"], big["faces"])
    assert not np.allclose(sm["points"], big["points"])
    tri = sm["points"][sm["faces"]].astype(np.float64)
    vol_s = np.einsum("ij,ij->i", tri[:, 0], np.cross(tri[:, 1], tri[:, 2])).sum() / 6
    assert abs(vol_s / (4 / 3 * np.pi * 20.0 ** 3) - 1) < 0.02   # Taubin keeps the volume
    with pytest.raises(ValueError, match="no surface at iso"):
        M.extract_surface(vol, (0, 0, 0), 1.0, 100.0)
    with pytest.raises(ValueError):
        M.extract_surface(vol, (0, 0, 0), 1.0, 0.0, decimate=0.5)
    path = M.save_mesh(sm, str(tmp_path / "bone.stl"))
    assert open(path, "rb").read(23) == b"minirecast surface (mm)"


def test_model_path_volume_otsu_surface(cuda):
    geom = circular_cone_vectors(90, 300.0, 600.0, 64, 80, 2.0)
    proj = oph.project_cone(oph.Phantom(scale=45.0), geom.vectors, 64, 80)
    rec = SliceReconstructor(proj, geom, verbose=False)
    vol, origin, h = rec.reconstruct_volume_tensor(maxdim=64)
    iso = M.otsu_threshold(vol)
    assert iso == om.otsu_threshold(vol.cpu().numpy())
    mesh = M.extract_surface(vol, origin, h, iso, smooth=0, min_piece=0.002)
    assert len(mesh["faces"]) > 100
    P, F = M.marching_cubes(vol, iso, origin, h)
    want_P, want_F = om.marching_cubes(vol.cpu().numpy(), iso, origin, h)
    np.testing.assert_array_equal(P.cpu().numpy(), want_P)
    np.testing.assert_array_equal(F.cpu().numpy(), want_F)
