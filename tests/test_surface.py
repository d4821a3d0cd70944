"""Iso-surface (model.extract_surface / marching_cubes, model.py:40-107) on the host side:
the library's own case table against the Python generator of the oracle, the oracle's
surfaces (closed, consistently oriented, Euler characteristic of a sphere, its area and
volume), and the STL writer. No reference output can be produced here (the reference
contours with VTK or scikit-image, neither installed), so the surface is checked by these
properties and the device path against the oracle (test_surface_gpu.py)."""
import ctypes
import struct

import numpy as np
import pytest

from oracle import mc_table as MT
from oracle import model as om
from tomography_local_demo_b200 import _native as N
from tomography_local_demo_b200 import model as M


def test_library_table_equals_python_generator():
    buf = (ctypes.c_int8 * (256 * 16))()
    assert N.load().mr_mc_table(buf) == N.MR_OK
    lib = np.frombuffer(buf, np.int8).reshape(256, 16)
    np.testing.assert_array_equal(lib[:, :15], MT.TRIANGLES)
    np.testing.assert_array_equal(lib[:, 15], MT.COUNTS)
    assert MT.COUNTS[0] == 0 and MT.COUNTS[255] == 0 and MT.COUNTS.max() == 5


def _closed_and_oriented(P, F):
    d = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
    und, cnt = np.unique(np.sort(d, axis=1), axis=0, return_counts=True)
    return bool(np.all(cnt == 2)) and len(np.unique(d, axis=0)) == len(d), len(P) - len(und) + len(F)


def sphere(n=40, r=12.0, centre=0.0):
    x = np.arange(n) - (n - 1) / 2 - centre
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    return (r - np.sqrt(X ** 2 + Y ** 2 + Z ** 2)).astype(np.float32)


def test_oracle_sphere_is_closed_and_measures_right():
    P, F = om.marching_cubes(sphere(), 0.0, origin=(-1.0, 2.0, 0.5), spacing=0.5)
    ok, euler = _closed_and_oriented(P, F)
    assert ok and euler == 2
    tri = P[F].astype(np.float64)
    volume = np.einsum("ij,ij->i", tri[:, 0], np.cross(tri[:, 1], tri[:, 2])).sum() / 6
    area = 0.5 * np.linalg.norm(np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0]), axis=1).sum()
    r = 12.0 * 0.5
    assert abs(volume / (4 / 3 * np.pi * r ** 3) - 1) < 0.01         # outward normals: volume > 0
    assert abs(area / (4 * np.pi * r ** 2) - 1) < 0.01


@pytest.mark.parametrize("seed", range(4))
def test_oracle_noise_surfaces_are_closed(seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(14, 12, 13)).astype(np.float32)
    v[0], v[-1], v[:, 0], v[:, -1], v[:, :, 0], v[:, :, -1] = -5, -5, -5, -5, -5, -5   # nothing on the border
    P, F = om.marching_cubes(v, 0.3)
    ok, _ = _closed_and_oriented(P, F)
    assert ok and len(F) > 0


def test_write_stl(tmp_path):
    P = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float)
    F = np.array([[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]])
    path = str(tmp_path / "m.stl")
    M.save_mesh({"points": P, "faces": F}, path)
    data = open(path, "rb").read()
    assert data[:23] == b"minirecast surface (mm)" and len(data) == 84 + 50 * 4
    assert struct.unpack("<I", data[80:84])[0] == 4
    n = np.frombuffer(data[84:84 + 12], "<f4")
    np.testing.assert_allclose(n, [0, 0, -1], atol=1e-7)
    with pytest.raises(SystemExit):
        M.save_mesh({"points": P, "faces": F}, str(tmp_path / "m.ply"))


def edge_crossing_vertices(vol, iso, origin, h):
    """The vertex set of an iso-contour as every marching-cubes variant emits it, the
    reference's contour included (model.py:54 VTK flying edges, model.py:72-75 scikit-image
    marching_cubes): one vertex on each grid edge whose end values lie on opposite sides of
    iso, at the linear interpolation point p0 + (iso - f0) / (f1 - f0) (p1 - p0), in float64.
    Written from that definition alone (no case table), so it pins the vertices of the
    surface to the reference's independently of the triangulation of ambiguous cells."""
    vol = np.asarray(vol, np.float64)
    out = []
    for axis in range(3):
        n = vol.shape[axis]
        f0 = np.take(vol, np.arange(n - 1), axis=axis)
        f1 = np.take(vol, np.arange(1, n), axis=axis)
        cross = (f0 < iso) != (f1 < iso)
        idx = np.argwhere(cross).astype(np.float64)
        t = (iso - f0[cross]) / (f1[cross] - f0[cross])
        idx[:, axis] += t
        out.append(np.asarray(origin, np.float64) + h * idx)
    return sorted_rows(np.concatenate(out))


def sorted_rows(P):
    P = np.asarray(P, np.float64)
    return P[np.lexsort(P.T[::-1])]


def assert_same_vertex_set(P, want, atol):
    """Every expected vertex has a distinct vertex of P within atol (nearest-neighbour
    matching: sorting FP32 and FP64 coordinates can order near-ties differently)."""
    from scipy.spatial import cKDTree
    P = np.asarray(P, np.float64)
    assert len(P) == len(want)
    d, idx = cKDTree(P).query(want)
    assert d.max() <= atol, (float(d.max()), atol)
    assert len(np.unique(idx)) == len(want)


@pytest.mark.parametrize("seed", [0, 1])
def test_oracle_vertices_are_the_contour_edge_crossings(seed):
    rng = np.random.default_rng(seed)
    vol = rng.normal(size=(13, 17, 11)).astype(np.float32)
    P, F = om.marching_cubes(vol, 0.1, (1.0, -2.0, 0.5), 0.7)
    want = edge_crossing_vertices(vol, 0.1, (1.0, -2.0, 0.5), 0.7)
    assert_same_vertex_set(P, want, 1e-5)
