"""Volume consumers of minirecast's model.py (model.py:18-29) on the device.

otsu_threshold(vol, bins=512) returns the reference's threshold bit for bit:
  v = vol[vol != 0]; lo, hi = np.percentile(v, [0.1, 99.95])
  hist = np.histogram(np.clip(v, lo, hi), bins, range=(lo, hi))
  argmax over the bins of w0 * w1 * (m0 - m1)^2 (Otsu's between-class variance)
The voxel passes run as CUDA kernels (mr_volume_stats / _select / _histogram: counts and
key range, exact order statistics by radix select, numpy's uniform-bin histogram of the
FP64-clipped values); the percentile interpolation between two order statistics and the
Otsu sums over the bins are host FP64 arithmetic on a few numbers, in numpy's order.
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
