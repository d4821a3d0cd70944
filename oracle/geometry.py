"""TEST INFRASTRUCTURE ONLY. NumPy restatement of minirecast's geometry helpers."""
import numpy as np


def circular_cone_vectors(n_angles, sod, sdd, pixel, angular_range=2 * np.pi, det_shift_u=0.0):
    """geometry.py:60-72 - ASTRA cone_vec rows of an ideal circular orbit about z."""
    vecs = np.zeros((n_angles, 12))
    for k in range(n_angles):
        a = k * angular_range / n_angles
        ray = np.array([np.cos(a), np.sin(a), 0.0])
        tan = np.array([-np.sin(a), np.cos(a), 0.0])
        vecs[k] = np.concatenate([-sod * ray, (sdd - sod) * ray + det_shift_u * pixel * tan,
                                  pixel * tan, [0.0, 0.0, pixel]])
    return vecs


def cone_volume_box(vectors, rows, cols):
    """geometry.py:49-57 - detector field of view at the axis, first view."""
    s, d, u, v = np.split(np.asarray(vectors, float)[0], 4)
    mag = np.linalg.norm(d - s) / np.linalg.norm(s)
    hu = cols * np.linalg.norm(u) / mag / 2.0
    return np.array([hu, hu, rows * np.linalg.norm(v) / mag / 2.0])


def parallel_volume_box(rows, cols, pixel_u, pixel_v):
    """geometry.py:29-34."""
    h = cols * pixel_u / 2.0
    return np.array([h, h, rows * pixel_v / 2.0])


def plane_basis(normal):
    """recon.py:225-235."""
    n = np.asarray(normal, dtype=float)
    n = n / np.linalg.norm(n)
    if abs(n[2]) < 0.9:
        e1 = np.cross([0.0, 0.0, 1.0], n)
    else:
        e1 = np.cross(n, [0.0, 1.0, 0.0])
    e1 = e1 / np.linalg.norm(e1)
    return n, e1, np.cross(n, e1)


def plane_size_for_box(box, normal):
    """recon.py:247-250."""
    _, e1, e2 = plane_basis(normal)
    return 2.0 * float(max(np.abs(e1) @ box, np.abs(e2) @ box))


def slice_points(box, origin, normal, n=256, size=None, zoom=1.0, center=None):
    """recon.py:238-265 (plane_points + slice_points)."""
    nh = np.asarray(normal, float) / np.linalg.norm(normal)
    c = np.zeros(3) if center is None else np.asarray(center, float)
    o = c - ((c - np.asarray(origin, float)) @ nh) * nh
    if size is None:
        size = plane_size_for_box(box, normal) / max(float(zoom), 1e-6)
    _, e1, e2 = plane_basis(normal)
    t = (np.arange(n) - (n - 1) / 2.0) * (size / n)
    a, b = np.meshgrid(t, t, indexing="xy")
    pts = o + a[..., None] * e1 + b[..., None] * e2
    return pts, np.all(np.abs(pts) <= box, axis=-1)


def volume_points(box, voxel=None, maxdim=None, native_pixel=None):
    """recon.py:278-283 + 449-460: (dims, origin, h) of the regular volume grid."""
    if maxdim is not None:
        h = 2.0 * float(np.max(box)) / maxdim
    else:
        h = float(voxel or native_pixel)
    dims = np.maximum(np.ceil(2.0 * np.asarray(box) / h).astype(int), 2)
    origin = -np.asarray(box) + h / 2.0
    return dims, origin, h


def arrival_order(n, mode="sequential"):
    """stream.py:12-29 - sequential or bit-reversed ("interleaved") acquisition order."""
    if mode == "sequential":
        return np.arange(n)
    if mode == "interleaved":
        bits = max(1, int(np.ceil(np.log2(n))))
        rev = np.array([int(format(i, f"0{bits}b")[::-1], 2) for i in range(2 ** bits)])
        return rev[rev < n]
    raise ValueError(f"unknown order {mode!r}")
