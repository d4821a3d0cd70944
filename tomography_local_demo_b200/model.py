"""Volume consumers of minirecast's model.py (model.py:18-107) on the device: the Otsu
threshold and the iso-surface (marching cubes) with its mesh export.

otsu_threshold(vol, bins=512) returns the reference's threshold bit for bit:
  v = vol[vol != 0]; lo, hi = np.percentile(v, [0.1, 99.95])
  hist = np.histogram(np.clip(v, lo, hi), bins, range=(lo, hi))
  argmax over the bins of w0 * w1 * (m0 - m1)^2 (Otsu's between-class variance)
The voxel passes run as CUDA kernels (mr_volume_stats / _select / _histogram: counts and
key range, exact order statistics by radix select, numpy's uniform-bin histogram of the
FP64-clipped values); the percentile interpolation between two order statistics and the
Otsu sums over the bins are host FP64 arithmetic on a few numbers, in numpy's order.

extract_surface / marching_cubes replace the VTK (or scikit-image) contour of
model.py:40-75 with two CUDA passes over the volume's cells (mr_mc_count, mr_mc_emit); the
reference's connectivity filter is a device label propagation, its smoothing a Taubin
lambda|mu pass; write_stl / save_mesh write the same binary STL as the reference.
"""
import ctypes

import numpy as np
import torch

from . import _native as N
from .recon import ctypes_void

PERCENTILES = (0.1, 99.95)          # the clip range of the reference (model.py:21)


def linear_neighbours(n, q):
    """numpy's "linear" percentile set-up for n sorted values (numpy 2.x): q / float32(100)
    in FP64, virtual index (n - 1) * q, neighbours floor(index) and floor(index) + 1 (the
    last value, rank n - 1, once the index reaches n - 1) and the blend weight
    g = index - floor(index) (numpy's own g, computed against -1 for the last value).
    Returns (prev ranks, next ranks, g), arrays over q."""
    if n < 1:
        raise IndexError("index -1 is out of bounds for axis 0 with size 0")
    q = np.true_divide(np.asarray(q, dtype=np.float64), np.float32(100))
    vi = (n - 1) * q
    prev = np.floor(vi)
    nxt = prev + 1
    above = vi >= n - 1
    prev[above] = -1
    nxt[above] = -1
    prev = prev.astype(np.intp)
    nxt = nxt.astype(np.intp)
    gamma = np.asarray(vi - prev, dtype=np.float64)
    return np.where(prev < 0, n - 1, prev), np.where(nxt < 0, n - 1, nxt), gamma


def lerp_like_numpy(a, b, gamma):
    """numpy's percentile blend of float32 neighbours a, b (broadcasting over gamma):
    their difference in FP32, then a + diff * g in FP64, or b - diff * (1 - g) for g >= 0.5."""
    a = np.asarray(a, dtype=np.float32)
    b = np.asarray(b, dtype=np.float32)
    gamma = np.asarray(gamma, dtype=np.float64)
    diff = np.subtract(b, a)                        # FP32
    return np.where(gamma >= 0.5, b - diff * (1 - gamma), a + diff * gamma)     # FP64


def percentile_linear(n, q, order_stat):
    """numpy.percentile(v, q) (method "linear", numpy 2.x) of n float32 values v, from
    order_stat(ranks) -> float32 values of those 0-based ascending ranks of v."""
    prev, nxt, gamma = linear_neighbours(n, q)
    ranks = np.unique(np.concatenate([prev, nxt]))
    vals = np.asarray(order_stat(ranks), dtype=np.float32)
    lookup = dict(zip(ranks.tolist(), vals))
    a = np.array([lookup[int(i)] for i in prev], dtype=np.float32)
    b = np.array([lookup[int(i)] for i in nxt], dtype=np.float32)
    return lerp_like_numpy(a, b, gamma)


def _device_volume(vol):
    if isinstance(vol, torch.Tensor):
        if vol.dtype != torch.float32:
            raise TypeError(f"otsu_threshold needs a float32 volume, got {vol.dtype}")
        t = vol if vol.is_cuda else vol.to(torch.device("cuda", torch.cuda.current_device()))
        return t.contiguous().reshape(-1)
    a = np.asarray(vol)
    if a.dtype != np.float32:
        raise TypeError(f"otsu_threshold needs a float32 volume, got {a.dtype}")
    dev = torch.device("cuda", torch.cuda.current_device())
    return torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).to(dev)


def otsu_threshold(vol, bins=512):
    """Otsu's threshold on the non-zero voxels (separates air from bone), model.py:18-29.
    vol: float32 volume, NumPy or torch (a CUDA tensor is used in place). Raises the
    reference's errors: IndexError when no voxel is non-zero, ValueError when the clip
    range is not finite (NaN or infinite voxels)."""
    bins = int(bins)
    if bins < 1 or bins > 2048:
        raise ValueError("bins must be in [1, 2048]")
    lib = N.load()
    t = _device_volume(vol)
    dev = t.device
    n = t.numel()
    v = ctypes_void
    with torch.cuda.device(dev):
        stream = torch.cuda.current_stream(dev)
        ws = torch.empty(int(lib.mr_volume_workspace_bytes()), dtype=torch.uint8, device=dev)
        stats = (ctypes.c_uint64 * 3)()
        N.check(lib.mr_volume_stats(v(t.data_ptr()) if n else None, n, v(ws.data_ptr()), stats,
                                    v(stream.cuda_stream)), "mr_volume_stats")
        nonzero, nan, keys = int(stats[0]), int(stats[1]), int(stats[2])
        if nan:
            raise ValueError("supplied range of [nan, nan] is not finite")
        kmin, kmax = keys & 0xFFFFFFFF, keys >> 32
        vals_dev = torch.empty(4, dtype=torch.float32, device=dev)

        def order_stat(ranks):
            r = (ctypes.c_int64 * len(ranks))(*[int(x) for x in ranks])
            N.check(lib.mr_volume_select(v(t.data_ptr()), n, r, len(ranks), kmin, kmax, v(ws.data_ptr()),
                                         v(vals_dev.data_ptr()), v(stream.cuda_stream)), "mr_volume_select")
            return vals_dev[:len(ranks)].cpu().numpy()

        lo, hi = percentile_linear(nonzero, PERCENTILES, order_stat)
        if not (np.isfinite(lo) and np.isfinite(hi)):
            raise ValueError(f"supplied range of [{lo}, {hi}] is not finite")
        first, last = lo, hi
        if first == last:                           # numpy widens an empty range
            first, last = first - 0.5, last + 0.5
        edges = np.linspace(first, last, bins + 1)
        edges_dev = torch.from_numpy(edges).to(dev)
        hist_dev = torch.empty(bins, dtype=torch.int64, device=dev)
        N.check(lib.mr_volume_histogram(v(t.data_ptr()), n, v(edges_dev.data_ptr()), bins, float(lo), float(hi),
                                        v(hist_dev.data_ptr()), v(stream.cuda_stream)), "mr_volume_histogram")
        hist = hist_dev.cpu().numpy().astype(np.intp)
    centers = 0.5 * (edges[1:] + edges[:-1])
    w0 = np.cumsum(hist)
    w1 = w0[-1] - w0
    m0 = np.cumsum(hist * centers) / np.maximum(w0, 1)
    m1 = (np.sum(hist * centers) - np.cumsum(hist * centers)) / np.maximum(w1, 1)
    between = w0 * w1 * (m0 - m1) ** 2
    return float(centers[int(np.argmax(between))])


# ------------------------------------------------------------------ surface
def marching_cubes(vol, iso, origin=(0.0, 0.0, 0.0), spacing=1.0):
    """Iso-surface of a float32 volume [nx, ny, nz] (grid point (i, j, k) at origin +
    spacing * (i, j, k)) on the device: (points f32 tensor [V, 3], faces int64 tensor [F, 3]),
    vertices shared between cells (one per crossed grid edge, in grid-edge order), faces in
    cell order, normals (right-hand rule) pointing from values above iso to values below.
    Two kernel passes (mr_mc_count, mr_mc_emit) with a scan of the per-block triangle
    counts between them; vertices are merged by the grid edge they lie on."""
    lib = N.load()
    t = vol if isinstance(vol, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(vol))
    if t.dtype != torch.float32 or t.dim() != 3:
        raise TypeError("marching_cubes needs a float32 volume [nx, ny, nz]")
    dev = t.device if t.is_cuda else torch.device("cuda", torch.cuda.current_device())
    t = t.to(dev).contiguous()
    nx, ny, nz = (int(d) for d in t.shape)
    v = ctypes_void
    with torch.cuda.device(dev):
        stream = torch.cuda.current_stream(dev)
        if min(nx, ny, nz) < 2:
            return (torch.zeros((0, 3), dtype=torch.float32, device=dev),
                    torch.zeros((0, 3), dtype=torch.int64, device=dev))
        nb = int(lib.mr_mc_blocks(nx, ny, nz))
        counts = torch.empty(nb, dtype=torch.int32, device=dev)
        N.check(lib.mr_mc_count(v(t.data_ptr()), nx, ny, nz, float(iso), v(counts.data_ptr()),
                                v(stream.cuda_stream)), "mr_mc_count")
        c64 = counts.to(torch.int64)
        offsets = torch.cumsum(c64, 0) - c64
        total = int(c64.sum())
        edges = torch.empty(3 * total, dtype=torch.int64, device=dev)
        pos = torch.empty((3 * total, 3), dtype=torch.float32, device=dev)
        org = (ctypes.c_double * 3)(*[float(x) for x in origin])
        N.check(lib.mr_mc_emit(v(t.data_ptr()), nx, ny, nz, float(iso), org, float(spacing), v(offsets.data_ptr()),
                               total, v(edges.data_ptr()) if total else None, v(pos.data_ptr()) if total else None,
                               v(stream.cuda_stream)), "mr_mc_emit")
        uniq, inv = torch.unique(edges, return_inverse=True)
        points = torch.empty((len(uniq), 3), dtype=torch.float32, device=dev)
        points[inv] = pos                       # every copy of a vertex holds the same value
        return points, inv.view(-1, 3)


def _components(faces, n_points):
    """Connected-component label (smallest vertex index) of every face: labels of a face's
    vertices are lowered to their minimum and chased to their roots until nothing changes."""
    label = torch.arange(n_points, device=faces.device)
    while True:
        m = label[faces].min(dim=1).values
        new = label.clone()
        for q in range(3):
            new.scatter_reduce_(0, faces[:, q], m, reduce="amin")
        new = new[new]
        if torch.equal(new, label):
            return label[faces[:, 0]]
        label = new


def _taubin(points, faces, n_iter, lam=0.5, mu=-0.53):
    """Taubin's lambda|mu smoothing with the uniform Laplacian over the mesh edges (keeps
    the volume, unlike plain Laplacian smoothing)."""
    e = torch.cat([faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [2, 0]]])
    e = torch.unique(torch.sort(e, dim=1).values, dim=0)
    a, b = e[:, 0], e[:, 1]
    deg = torch.zeros(len(points), dtype=points.dtype, device=points.device)
    deg.index_add_(0, a, torch.ones_like(a, dtype=points.dtype))
    deg.index_add_(0, b, torch.ones_like(b, dtype=points.dtype))
    deg = deg.clamp(min=1.0)[:, None]
    p = points.clone()
    for _ in range(int(n_iter)):
        for f in (lam, mu):
            s = torch.zeros_like(p)
            s.index_add_(0, a, p[b])
            s.index_add_(0, b, p[a])
            p = p + f * (s / deg - p)
    return p


def extract_surface(vol, origin, spacing, iso, smooth=15, min_piece=0.002, decimate=0.0):
    """Iso-surface of the volume (model.py:40-69), as the reference's scikit-image fallback
    returns it: dict(points [V, 3] float32, faces [F, 3] int64). The contour is marching
    cubes on the device; min_piece drops the connected pieces with fewer than that fraction
    of the triangles (the reference's connectivity filter); smooth > 0 runs that many Taubin
    lambda|mu iterations (the reference calls VTK's windowed-sinc variant). Decimation is
    not provided here (decimate must be 0)."""
    if decimate and float(decimate) > 0:
        raise ValueError("decimation is not provided by this library: use decimate=0")
    points, faces = marching_cubes(vol, iso, origin, spacing)
    if len(faces) == 0:
        raise ValueError(f"no surface at iso={iso:g}; try a lower --iso")
    if min_piece > 0:
        ids = _components(faces, len(points))
        uniq, inv, counts = torch.unique(ids, return_inverse=True, return_counts=True)
        keep = counts[inv] >= min_piece * len(ids)
        faces = faces[keep]
        used, faces = torch.unique(faces, return_inverse=True)
        points = points[used]
    if smooth and int(smooth) > 0:
        points = _taubin(points, faces, int(smooth))
    return {"points": points.cpu().numpy(), "faces": faces.cpu().numpy()}


def mesh_arrays(mesh):
    """(points [n, 3], triangles [m, 3]) of a mesh dict (model.py:78-83)."""
    return mesh["points"], mesh["faces"]


def write_stl(path, points, faces):
    """Binary STL in mm (model.py:86-96): 80-byte header, triangle count, then per triangle
    the unit normal, three vertices (float32) and a zero attribute word."""
    import struct
    points = np.asarray(points, dtype=np.float64)
    faces = np.asarray(faces)
    tri = points[faces]
    n = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-12)
    rec = np.zeros(len(faces), dtype=[("n", "<f4", 3), ("v", "<f4", (3, 3)), ("a", "<u2")])
    rec["n"], rec["v"] = n, tri
    with open(path, "wb") as f:
        f.write(b"minirecast surface (mm)".ljust(80, b" "))
        f.write(struct.pack("<I", len(faces)))
        f.write(rec.tobytes())


def save_mesh(mesh, path):
    """Write a mesh dict to .stl (model.py:99-107; the reference writes other formats
    through pyvista, which this package does not use)."""
    import os
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    if path.lower().endswith(".stl"):
        write_stl(path, *mesh_arrays(mesh))
    else:
        raise SystemExit("without pyvista only .stl export is available")
    return path
