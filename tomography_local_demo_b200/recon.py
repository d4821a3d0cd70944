"""On-demand slice reconstruction on one B200: the drop-in for minirecast recon.py.

Projections are filtered on arrival (FBP / FDK row filter, sm_100a FFT kernel) into a
device-resident ring of filtered views; any slice, point set or volume is then
back-projected on demand by the sm_100a voxel-driven kernel from every view received
so far. The public surface (module functions and `SliceReconstructor`) follows
minirecast recon.py:34-519 name for name; NumPy in, NumPy out, with torch-tensor
variants for device-resident callers.

FP64 is used on the host only, to build the per-view projective maps and the filter
spectrum (as the reference does); the device computes in FP32 and stores the filtered
views in FP32 (default), BF16 or FP16.
"""
import collections
import ctypes
import threading
import time

import numpy as np
import torch

from . import _native as N
from . import preprocess
from .geometry import ConeVecGeometry, ParallelGeometry

HAVE_CUDA = True
BACKEND = "cuda-sm100a"

_STORE_DTYPES = {"fp32": (N.MR_F32, torch.float32), "bf16": (N.MR_BF16, torch.bfloat16),
                 "fp16": (N.MR_F16, torch.float16)}


def ring_pitch(cols, store="fp32"):
    """Row pitch (elements) of the filtered-view ring: the smallest multiple of 32 bytes
    that holds `cols` values, so that every row starts 32-byte aligned and the tensor-core
    filter stores each view's row in 32-byte pieces (16-byte pieces on a misaligned row
    cost a quarter of its time: 0.309 against 0.288 ms for 600 views of 486 x 384)."""
    per = 32 // torch.empty((), dtype=_STORE_DTYPES[store][1]).element_size()
    return (int(cols) + per - 1) // per * per


# --------------------------------------------------------------------------
# Filter spectrum (host, FP64) - recon.py:34-55
# --------------------------------------------------------------------------
def ramp_response(n, tau, window="shepp-logan"):
    """Spectrum of the discrete Ram-Lak kernel (Kak & Slaney), zero-padded to
    N = 2^ceil(log2(2n)), times an optional apodisation window. Returns (H, N)."""
    N_fft = int(2 ** np.ceil(np.log2(2 * n)))
    m = np.fft.fftfreq(N_fft, d=1.0 / N_fft).astype(np.int64)     # 0..N/2-1, -N/2..-1
    h = np.zeros(N_fft)
    h[0] = 1.0 / (4.0 * tau * tau)
    odd = m % 2 == 1
    h[odd] = -1.0 / (np.pi * m[odd] * tau) ** 2
    H = np.real(np.fft.fft(h)) * tau
    f = np.fft.fftfreq(N_fft)
    if window in (None, "ram-lak", "none"):
        pass
    elif window == "shepp-logan":
        H *= np.sinc(f)
    elif window == "hann":
        H *= 0.5 * (1.0 + np.cos(2.0 * np.pi * f))
    elif window == "cosine":
        H *= np.cos(np.pi * f)
    else:
        raise ValueError(f"unknown filter window {window!r}")
    return H, N_fft


class _FilterTables:
    """Device copies of the tau = 1 spectrum (mirrored from the rfft half, exactly the
    bins irfft uses) and of the FFT twiddles, for one detector width and window."""

    def __init__(self, cols, window, device):
        H, n_fft = ramp_response(cols, 1.0, window)
        half = H[: n_fft // 2 + 1]
        full = np.concatenate([half, half[1:n_fft - n_fft // 2][::-1]])
        tw = np.exp(-2j * np.pi * np.arange(n_fft) / n_fft)
        self.n_fft = n_fft
        self.log2n = int(round(np.log2(n_fft)))
        self.H = torch.from_numpy(full.astype(np.float32)).to(device)
        self.tw = torch.from_numpy(np.stack([tw.real, tw.imag], 1).astype(np.float32)).to(device)
        self._full64 = full
        self._cols = cols
        self._device = device
        self._tc_image = {}

    def tc_image(self, fmt=None):
        """(device operand, t_scale) of the tensor-core Toeplitz filter (mr_toeplitz_image):
        the split FP16 (default) or BF16 blocks of g = ifft(H) (tau = 1, FP64 on the host),
        built on first use."""
        fmt = N.MR_F16 if fmt is None else fmt
        if fmt not in self._tc_image:
            lib = N.load()
            nbytes = lib.mr_toeplitz_image_bytes(self._cols)
            if nbytes < 0:
                raise ValueError(f"the tensor-core filter supports rows of at most 512 columns, not {self._cols}")
            g = np.ascontiguousarray(np.fft.ifft(self._full64).real, dtype=np.float64)
            img = np.zeros(nbytes, dtype=np.uint8)
            ts = ctypes.c_float()
            N.check(lib.mr_toeplitz_image(g.ctypes.data, self.n_fft, self._cols, fmt, img.ctypes.data,
                                          ctypes.byref(ts)), "mr_toeplitz_image")
            self._tc_image[fmt] = (torch.from_numpy(img).to(self._device), float(ts.value))
        return self._tc_image[fmt]


# --------------------------------------------------------------------------
# Per-view constants (host, FP64) - recon.py:70-82
# --------------------------------------------------------------------------
def cone_constants(vectors):
    """Per view: src, det, u, v, u/|u|^2, v/|v|^2, unit normal oriented source ->
    detector, source-detector-plane distance SDD and source-axis distance SOD."""
    V = np.asarray(vectors, dtype=np.float64)
    s, d, u, v = V[:, 0:3], V[:, 3:6], V[:, 6:9], V[:, 9:12]
    n = np.cross(u, v)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    n *= np.sign(np.einsum("ij,ij->i", d - s, n))[:, None]
    sdd = np.einsum("ij,ij->i", d - s, n)
    sod = np.einsum("ij,ij->i", -s, n)
    uu = u / np.einsum("ij,ij->i", u, u)[:, None]
    vv = v / np.einsum("ij,ij->i", v, v)[:, None]
    return dict(s=s, d=d, u=u, v=v, uu=uu, vv=vv, n=n, sdd=sdd, sod=sod)


def cone_view_maps(K, rows, cols, qscale=None):
    """FP64 projective maps of cone views -> mr_view records (FP32).

    With L = (p - s).n, t = SDD/L and X = s + t (p - s) - d (recon.py:206-215):
    col = X.uu + (C-1)/2 = (pu.[p,1]) / den, row likewise, den = L / SOD, so the FDK
    weight (SOD/L)^2 is 1/den^2."""
    s, d, n, uu, vv = K["s"], K["d"], K["n"], K["uu"], K["vv"]
    sdd, sod = K["sdd"][:, None], K["sod"][:, None]
    e_u = np.einsum("ij,ij->i", s - d, uu)[:, None] + (cols - 1) / 2.0
    e_v = np.einsum("ij,ij->i", s - d, vv)[:, None] + (rows - 1) / 2.0
    n_s = np.einsum("ij,ij->i", n, s)[:, None]
    out = np.zeros(len(s), dtype=N.VIEW_DTYPE)
    pu = np.concatenate([(e_u * n + sdd * uu) / sod,
                         -(e_u * n_s + sdd * np.einsum("ij,ij->i", uu, s)[:, None]) / sod], 1)
    pv = np.concatenate([(e_v * n + sdd * vv) / sod,
                         -(e_v * n_s + sdd * np.einsum("ij,ij->i", vv, s)[:, None]) / sod], 1)
    pw = np.concatenate([n / sod, -n_s / sod], 1)
    out["pu"], out["pv"], out["pw"] = pu, pv, pw
    out["uv"] = np.einsum("ij,ij->i", K["u"], vv)
    out["qscale"] = 1.0 if qscale is None else qscale
    return out


def parallel_view_maps(angles, pixel_u, pixel_v, rows, cols, qscale=None):
    """Affine maps of parallel views (recon.py:185-188): col = (-x sin + y cos)/pu +
    (C-1)/2, row = z/pv + (R-1)/2, den = 1."""
    a = np.asarray(angles, dtype=np.float64)
    out = np.zeros(len(a), dtype=N.VIEW_DTYPE)
    out["pu"][:, 0] = -np.sin(a) / pixel_u
    out["pu"][:, 1] = np.cos(a) / pixel_u
    out["pu"][:, 3] = (cols - 1) / 2.0
    out["pv"][:, 2] = 1.0 / pixel_v
    out["pv"][:, 3] = (rows - 1) / 2.0
    out["pw"][:, 3] = 1.0
    out["qscale"] = 1.0 if qscale is None else qscale
    return out


def parker_weights(vectors, cols):
    """Short-scan weights w[v, c] of D. L. Parker (Med. Phys. 9, 254-257, 1982) for a circular
    cone-beam orbit, FP64 [views, cols].

    beta = source angle from the first view along the orbit, gamma = fan angle of column c
    in the mid-plane, measured from the central ray (source -> rotation axis) in the
    direction of rotation, so that the ray (beta, gamma) is measured again at
    (beta + pi + 2 gamma, -gamma). With 2 delta = (last beta) - pi:
      w = sin^2(pi/4 * beta / (delta - gamma))               0 <= beta < 2 (delta - gamma)
      w = 1                                                   up to beta = pi - 2 gamma
      w = sin^2(pi/4 * (pi + 2 delta - beta) / (delta + gamma))  up to beta = pi + 2 delta
    so that every ray's two measurements weigh 1 together. The weights are multiplied by
    n d_beta / pi, which keeps the back-projection's FDK scale pi / n right for the weighted
    short scan (a full scan has no such scale: each ray counts twice with weight 1 / 2)."""
    V = np.asarray(vectors, dtype=np.float64)
    n = len(V)
    if n < 3:
        raise ValueError("Parker weights need at least 3 views")
    s, d, u = V[:, 0:3], V[:, 3:6], V[:, 6:9]
    th = np.unwrap(np.arctan2(s[:, 1], s[:, 0]))
    sigma = 1.0 if th[-1] >= th[0] else -1.0
    beta = sigma * (th - th[0])
    d_beta = beta[-1] / (n - 1)
    if beta[-1] + 1.5 * d_beta >= 2 * np.pi:
        raise ValueError("Parker weights are for short scans: this orbit covers a full turn")
    off = np.arange(cols) - (cols - 1) / 2.0
    ray = d[:, None, :] + off[None, :, None] * u[:, None, :] - s[:, None, :]       # [n, C, 3]
    cen = -s
    gamma = sigma * np.arctan2(cen[:, None, 0] * ray[..., 1] - cen[:, None, 1] * ray[..., 0],
                               cen[:, None, 0] * ray[..., 0] + cen[:, None, 1] * ray[..., 1])
    delta = (beta[-1] - np.pi) / 2.0
    if delta <= np.abs(gamma).max():
        raise ValueError(f"the orbit covers {np.degrees(beta[-1]):.1f} deg: a short scan needs 180 deg "
                         f"plus the fan angle ({np.degrees(2 * np.abs(gamma).max()):.1f} deg)")
    b = beta[:, None]
    w = np.ones_like(gamma)
    lo = b < 2.0 * (delta - gamma)
    hi = b > np.pi - 2.0 * gamma
    w[lo] = np.sin(np.pi / 4.0 * (b / (delta - gamma))[lo]) ** 2
    w[hi] = np.sin(np.pi / 4.0 * ((np.pi + 2.0 * delta - b) / (delta + gamma))[hi]) ** 2
    return w * (n * d_beta / np.pi)


def cone_filter_views(K, rows, cols, n_fft, slots, out_scale=1.0):
    """mr_filter_view records of cone views (fdk_filter_block, recon.py:93-103)."""
    s, d, u, v, n = K["s"], K["d"], K["u"], K["v"], K["n"]
    sdd, sod = K["sdd"], K["sod"]
    off = d - (s + sdd[:, None] * n)
    un, vn = np.linalg.norm(u, axis=1), np.linalg.norm(v, axis=1)
    fv = np.zeros(len(s), dtype=N.FILTER_VIEW_DTYPE)
    fv["a0"] = np.einsum("ij,ij->i", off, u) / un - (cols - 1) / 2.0 * un
    fv["da"] = un
    fv["b0"] = np.einsum("ij,ij->i", off, v) / vn - (rows - 1) / 2.0 * vn
    fv["db"] = vn
    fv["sdd"] = sdd
    tau = un * sod / sdd
    fv["gain"] = 1.0 / (tau * n_fft)
    fv["out_scale"] = out_scale
    fv["slot"] = slots
    return fv


def parallel_filter_views(pixel_u, k, n_fft, slots, out_scale=1.0):
    fv = np.zeros(k, dtype=N.FILTER_VIEW_DTYPE)
    fv["gain"] = 1.0 / (pixel_u * n_fft)
    fv["out_scale"] = out_scale
    fv["slot"] = slots
    return fv


# --------------------------------------------------------------------------
# Device helpers
# --------------------------------------------------------------------------
# |-log(max(t, 1e-3))| of corrected raw counts stays below 11.1 when t <= 65535 (FleX-ray
# gain 1 / max(F - D, 1)); the tensor-core input scale it gives (1024, as in the fused raw
# ingest) keeps any |x| < 64 inside FP16's range, which covers the HDF5 gain
# 1 / max(F - D, 1e-6) too (|x| < 25)
RAW_LINE_BOUND = 11.1


def _device(device=None):
    if not torch.cuda.is_available():
        raise RuntimeError("a CUDA device is required: this library has no CPU path")
    return torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)


def ctypes_void(x):
    import ctypes
    return ctypes.c_void_p(int(x))


def _ring_struct(ring_tensor, dtype_code, kind, rows, cols):
    r = N.MrRing()
    r.data = ring_tensor.data_ptr()
    r.dtype = dtype_code
    r.kind = kind
    r.rows = rows
    r.cols = cols
    r.col_pitch = ring_tensor.shape[2]
    r.n_slots = ring_tensor.shape[0]
    r.slot_stride = ring_tensor.shape[1] * ring_tensor.shape[2]
    return r


def _to_device_tensor(arr, device, dtype=None):
    if isinstance(arr, torch.Tensor):
        t = arr
    else:
        t = torch.from_numpy(np.ascontiguousarray(arr))
    if dtype is not None:
        t = t.to(dtype)
    return t.to(device, non_blocking=True).contiguous()


def _handoff(stream, *tensors):
    """Order the caller's current stream after `stream` (where `tensors` were produced)
    and tell the allocator the tensors are used there, so results returned by the
    *_tensor methods are safe to use on the caller's stream."""
    cur = torch.cuda.current_stream(stream.device)
    if cur.cuda_stream != stream.cuda_stream:
        ev = torch.cuda.Event()
        ev.record(stream)
        cur.wait_event(ev)
        for t in tensors:
            t.record_stream(cur)


class _RecordStaging:
    """Page-locked staging for the small records that go up with every launch: a ring of
    fixed slots reused in turn, each guarded by the event of its last copy, so the host
    runs at most `slots` uploads ahead of the GPU. Taking page-locked memory per call
    instead grows torch's host cache whenever the host runs ahead, and single allocations
    of that cache took up to 3.5 ms, stalling the launching thread."""

    def __init__(self, slots=32, slot_bytes=128 << 10):
        self.slot_bytes = slot_bytes
        self.buf = torch.empty(slots * slot_bytes, dtype=torch.uint8).pin_memory()
        self.host = self.buf.numpy()
        self.events = [None] * slots
        self.next = 0
        self.lock = threading.Lock()

    def upload(self, raw, device, out=None):
        """Device copy of the uint8 array `raw` on the current stream (asynchronous), into
        `out` when given, or None when it does not fit a slot."""
        n = raw.size
        if n > self.slot_bytes:
            return None
        with self.lock:
            k = self.next
            self.next = (k + 1) % len(self.events)
            if self.events[k] is not None:
                self.events[k].synchronize()         # the slot's previous copy has run
            o = k * self.slot_bytes
            self.host[o:o + n] = raw
            dst = torch.empty(n, dtype=torch.uint8, device=device) if out is None else out
            dst.copy_(self.buf[o:o + n], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(torch.cuda.current_stream(device))
            self.events[k] = ev
        return dst


_STAGING = {}
_STAGING_LOCK = threading.Lock()


def _staging(device):
    """The record staging ring of `device` (created on first use)."""
    key = torch.device(device).index
    with _STAGING_LOCK:
        if key not in _STAGING:
            _STAGING[key] = _RecordStaging()
        return _STAGING[key]


def _struct_tensor(records, device, asynchronous=False):
    """Device copy of numpy ABI records on the current stream. By default a small pageable
    copy, which the host waits for but which is not queued behind large pinned transfers
    that other streams have in flight; asynchronous=True stages it in page-locked memory
    instead, so the host does not wait (for when no such transfer is in flight)."""
    raw = np.ascontiguousarray(records).view(np.uint8).reshape(-1)
    if asynchronous:
        dst = _staging(device).upload(raw, device)
        if dst is not None:
            return dst
        return torch.from_numpy(raw.copy()).pin_memory().to(device, non_blocking=True)
    return torch.from_numpy(raw.copy()).to(device, non_blocking=False)


def filter_block_device(block, s_view, s_row, k, fviews_dev, tables, ring, stream, method="fft", status=None,
                        x_bound=None):
    """Filter k views of a device f32 block into ring slots: mr_filter_f32 (FFT) or
    mr_filter_f32_tc (tensor-core Toeplitz GEMM, split FP16 "tc" or split BF16 "tc-bf16").
    x_bound: a known bound on |block| (the tensor-core input scale is then set from it,
    without reading the block back to the host)."""
    lib = N.load()
    if method in ("tc", "tc-bf16"):
        fmt = N.MR_BF16 if method == "tc-bf16" else N.MR_F16
        img, t_scale = tables.tc_image(fmt)
        # power of two with max |x| * x_scale in [2^13, 2^14) (FP16 range for the hi part)
        if x_bound is not None:
            m = float(x_bound)
        else:
            m = float(block.abs().amax()) if block.numel() else 0.0
        x_scale = 2.0 ** int(np.clip(14 - np.frexp(m)[1], -100, 100)) if m > 0 and np.isfinite(m) else 1.0
        st = lib.mr_filter_f32_tc(ctypes_void(block.data_ptr()), s_view, s_row, k,
                                  ctypes_void(fviews_dev.data_ptr()), ctypes_void(img.data_ptr()), fmt, t_scale,
                                  x_scale, tables.n_fft, ring,
                                  ctypes_void(status.data_ptr()) if status is not None else None,
                                  ctypes_void(stream.cuda_stream))
        N.check(st, "mr_filter_f32_tc")
        return
    st = lib.mr_filter_f32(ctypes_void(block.data_ptr()), s_view, s_row, k,
                           ctypes_void(fviews_dev.data_ptr()), ctypes_void(tables.H.data_ptr()),
                           ctypes_void(tables.tw.data_ptr()), tables.log2n, ring,
                           ctypes_void(stream.cuda_stream))
    N.check(st, "mr_filter_f32")


class KernelTimer:
    """CUDA events recorded right around each library launch, on the launch's stream."""

    def __init__(self):
        self.records = []

    def start(self, stream):
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(stream)
        return ev

    def stop(self, name, ev0, stream):
        ev1 = torch.cuda.Event(enable_timing=True)
        ev1.record(stream)
        self.records.append((name, ev0, ev1))

    def summary(self):
        """{name: (launches, total ms)} of everything recorded so far."""
        torch.cuda.synchronize()
        out = {}
        for name, a, b in self.records:
            n, t = out.get(name, (0, 0.0))
            out[name] = (n + 1, t + a.elapsed_time(b))
        return out

    def clear(self):
        self.records = []


def backproject_device(ring, views_dev, grids, out, stream, device, timer=None, kernel="staged",
                       status=None, wait=None, asynchronous=False, band_axis=None):
    """Back-project numpy GRID_DTYPE records into the device f32 tensor `out`.

    kernel="staged": regular grids go through mr_backproject_staged (TMA-staged
    footprints); point lists always use mr_backproject. kernel="plain": everything uses
    mr_backproject (direct global gathers) - the plain GPU path kept for comparison.
    wait: an event the launch must follow (the filter of the views summed); the grid and
    tile records are uploaded before the stream waits for it (asynchronously from
    page-locked memory with asynchronous=True). band_axis: the orbit's rotation axis, which
    orders the tiles of regular grids by height (_native.plan_tiles)."""
    grids = np.ascontiguousarray(grids, dtype=N.GRID_DTYPE)
    is_pts = (grids["flags"] & N.MR_GRID_POINTS) != 0
    if kernel == "staged" and is_pts.any() and not is_pts.all():
        backproject_device(ring, views_dev, grids[is_pts], out, stream, device, timer, "plain", wait=wait,
                           asynchronous=asynchronous)
        wait = None
        grids = grids[~is_pts]
        is_pts = is_pts[~is_pts]
    tiles = N.plan_tiles(grids, band_axis)
    if len(tiles) == 0:
        if wait is not None:
            stream.wait_event(wait)
        return
    # grid and tile records in one upload (the grid records are 256 bytes each, so the
    # tiles that follow them stay aligned)
    recs = _struct_tensor(np.concatenate([grids.view(np.uint8), tiles.view(np.uint8)]), device, asynchronous)
    g_ptr, t_ptr = recs.data_ptr(), recs.data_ptr() + grids.nbytes
    if wait is not None:
        stream.wait_event(wait)
    lib = N.load()
    v = ctypes_void
    staged = kernel == "staged" and not is_pts.any()
    name = "mr_backproject_staged" if staged else "mr_backproject"
    ev0 = timer.start(stream) if timer is not None else None
    if staged:
        st = lib.mr_backproject_staged(ring, v(views_dev.data_ptr()), v(g_ptr), v(t_ptr),
                                       len(tiles), v(out.data_ptr()),
                                       v(status.data_ptr()) if status is not None else None,
                                       v(stream.cuda_stream))
    else:
        st = lib.mr_backproject(ring, v(views_dev.data_ptr()), v(g_ptr), v(t_ptr),
                                len(tiles), v(out.data_ptr()), v(stream.cuda_stream))
    if timer is not None:
        timer.stop(name, ev0, stream)
    N.check(st, name)
    # keep the descriptor tensor alive until the kernel has consumed it
    recs.record_stream(stream)


# --------------------------------------------------------------------------
# Stand-alone filter functions (recon.py:58-64, 85-104), run on the GPU
# --------------------------------------------------------------------------
def _filter_generic(data3, fviews, cols, window, device):
    """data3: [k, R, C] f32 -> [k, R, C] f32 filtered on the device."""
    dev = _device(device)
    k, R, C = data3.shape
    tables = _FilterTables(C, window, dev)
    pitch = (C + 7) // 8 * 8
    with torch.cuda.device(dev):
        stream = torch.cuda.current_stream(dev)
        x = _to_device_tensor(np.ascontiguousarray(data3, dtype=np.float32), dev)
        out = torch.empty((k, R, pitch), dtype=torch.float32, device=dev)
        ring = _ring_struct(out, N.MR_F32, N.MR_PARALLEL, R, C)
        fv = fviews(tables.n_fft)
        fv_dev = _struct_tensor(fv, dev)
        for v0 in range(0, k, 65535):
            kk = min(65535, k - v0)
            sub = x[v0:v0 + kk]
            fv_sub = fv_dev[v0 * N.FILTER_VIEW_DTYPE.itemsize:(v0 + kk) * N.FILTER_VIEW_DTYPE.itemsize]
            filter_block_device(sub, R * C, C, kk, fv_sub, tables, ring, stream)
        res = out[:, :, :C].cpu().numpy()
    return res


def filter_rows(data, tau, window="shepp-logan"):
    """Ramp-filter along the last axis (any leading shape), FP32 FFT on the device."""
    a = np.asarray(data, dtype=np.float32)
    shape = a.shape
    C = shape[-1]
    flat = a.reshape(-1, 1, C)
    k = flat.shape[0]
    res = _filter_generic(flat, lambda n_fft: parallel_filter_views(tau, k, n_fft, np.arange(k)),
                          C, window, None)
    return res.reshape(shape)


def fdk_filter_block(block, K, window="shepp-logan"):
    """FDK cosine pre-weight + ramp filter of block [rows, k, cols] -> [k, rows, cols]."""
    b = np.asarray(block, dtype=np.float32)
    R, A, C = b.shape
    data3 = np.ascontiguousarray(np.transpose(b, (1, 0, 2)))
    return _filter_generic(data3, lambda n_fft: cone_filter_views(K, R, C, n_fft, np.arange(A)),
                           C, window, None)


# --------------------------------------------------------------------------
# Plane helpers (host, FP64) - recon.py:225-283
# --------------------------------------------------------------------------
def _cross3(a, b):
    """a x b of two 3-vectors with numpy.cross's arithmetic (each component one product
    minus another, rounded the same way) at a fraction of its call overhead."""
    a0, a1, a2 = float(a[0]), float(a[1]), float(a[2])
    b0, b1, b2 = float(b[0]), float(b[1]), float(b[2])
    return np.array([a1 * b2 - a2 * b1, a2 * b0 - a0 * b2, a0 * b1 - a1 * b0])


def plane_basis(normal):
    n = np.asarray(normal, dtype=float)
    n = n / np.linalg.norm(n)
    z = np.array([0.0, 0.0, 1.0])
    e1 = _cross3(z, n) if abs(n @ z) < 0.9 else _cross3(n, (0.0, 1.0, 0.0))
    e1 /= np.linalg.norm(e1)
    return n, e1, _cross3(n, e1)


def plane_points(origin, normal, size, n):
    """n x n points (mm) of a square of side `size`: rows follow e2, columns e1."""
    _, e1, e2 = plane_basis(normal)
    t = (np.arange(n) - (n - 1) / 2.0) * (size / n)
    a, b = np.meshgrid(t, t, indexing="xy")
    return np.asarray(origin, float) + a[..., None] * e1 + b[..., None] * e2


def plane_size_for_box(box, normal, basis=None):
    _, e1, e2 = plane_basis(normal) if basis is None else basis
    return 2.0 * float(max(np.abs(e1) @ box, np.abs(e2) @ box))


def _plane_frame(box, origin, normal, n, size, zoom, center):
    """(centre on the plane, e1, e2, size) as computed by slice_points."""
    n_hat = np.asarray(normal, float) / np.linalg.norm(normal)
    o = np.asarray(origin, float)
    c = np.zeros(3) if center is None else np.asarray(center, float)
    o = c - ((c - o) @ n_hat) * n_hat
    basis = plane_basis(normal)
    if size is None:
        size = plane_size_for_box(box, normal, basis) / max(float(zoom), 1e-6)
    return o, basis[1], basis[2], float(size)


def slice_points(box, origin, normal, n=256, size=None, zoom=1.0, center=None):
    """Points of an n x n slice and its in-box mask (recon.py:253-265)."""
    o, _, _, size = _plane_frame(box, origin, normal, n, size, zoom, center)
    pts = plane_points(o, normal, size, n)
    mask = np.all(np.abs(pts) <= box, axis=-1)
    return pts, mask


def planes_intersection(normals, origins, fallback=(0.0, 0.0, 0.0)):
    N_ = np.asarray(normals, float)
    N_ = N_ / np.linalg.norm(N_, axis=1, keepdims=True)
    b = np.einsum("ij,ij->i", N_, np.asarray(origins, float))
    if np.linalg.matrix_rank(N_, tol=1e-3) < 3:
        return np.asarray(fallback, float)
    return np.linalg.lstsq(N_, b, rcond=None)[0]


def volume_grid(box, maxdim):
    h = 2.0 * float(np.max(box)) / maxdim
    dims = np.maximum(np.ceil(2.0 * np.asarray(box) / h).astype(int), 2)
    origin = -np.asarray(box) + h / 2.0
    return dims, origin, h


def plane_grid(box, origin, normal, n, size=None, zoom=1.0, center=None, cor_shift=0.0):
    """One mr_grid record for an n x n slice (masked to the box), output offset 0."""
    o, e1, e2, size = _plane_frame(box, origin, normal, n, size, zoom, center)
    g = np.zeros(1, dtype=N.GRID_DTYPE)[0]
    delta = size / n
    half = (n - 1) / 2.0
    t0 = -half * delta
    g["origin"] = o + t0 * e1 + t0 * e2
    g["step_i"] = delta * e2
    g["step_j"] = delta * e1
    g["cor_shift"] = cor_shift
    g["n_i"], g["n_j"], g["n_k"] = n, n, 1
    g["flags"] = N.MR_GRID_MASK_BOX
    g["out_stride_i"], g["out_stride_j"] = n, 1
    g["mask_c"], g["mask_ej"], g["mask_ei"] = o, e1, e2
    g["mask_half"], g["mask_delta"] = half, delta
    g["box"] = box
    return g


def volume_grid_record(origin, h, dims, k0=0, k1=None):
    """mr_grid record of a regular volume [nx, ny, nz] (x slowest, z fastest), for the
    x planes [k0, k1): samples (i=y, j=z, k=x)."""
    nx, ny, nz = (int(d) for d in dims)
    k1 = nx if k1 is None else k1
    g = np.zeros(1, dtype=N.GRID_DTYPE)[0]
    g["origin"] = [origin[0] + h * k0, origin[1], origin[2]]
    g["step_i"] = [0.0, h, 0.0]
    g["step_j"] = [0.0, 0.0, h]
    g["step_k"] = [h, 0.0, 0.0]
    g["n_i"], g["n_j"], g["n_k"] = ny, nz, k1 - k0
    g["out_offset"] = k0 * ny * nz
    g["out_stride_i"], g["out_stride_j"], g["out_stride_k"] = nz, 1, ny * nz
    return g


# --------------------------------------------------------------------------
# Public reconstructor (recon.py:289-519)
# --------------------------------------------------------------------------
class SliceReconstructor:
    """Filter projections as they arrive, then reconstruct any slice on demand.

    proj     : optional [rows, angles, cols] array with ALL projections (batch mode);
               omit it and call add_projections() to stream data in (live mode).
    gaussian : sigma (detector pixels) of a Gaussian low-pass on each projection.
    tilt     : detector tilt correction in degrees (rotates each projection).
    store    : filtered-view storage, "fp32" (default), "bf16" or "fp16".
    device   : CUDA device (default: the current one).
    keep_projections : also keep the unfiltered (pre-processed) line integrals of every
               received view on the device (FP32, the ring's layout), for refine_slice_ls.
    filter   : "fft" (default; shared-memory FFT, FP32), "tc" (Toeplitz GEMM on the tensor
               cores, split FP16 operands, FP32 accumulation; rows <= 512 columns) or
               "tc-bf16" (the same with split BF16 operands, ~100x less precise on
               smooth rows because the ramp filter cancels strongly).
    parker   : weight a cone-beam short scan (180 deg plus the fan angle, up to a full turn)
               with Parker's weights before the filter; the reference has no such weights
               and only warns (recon.py:331-332).
    The `backend` argument is accepted for compatibility; the backend is always
    "cuda-sm100a".
    """

    def __init__(self, proj=None, geom=None, window="shepp-logan", backend="auto",
                 gaussian=0.0, tilt=0.0, verbose=True, store="fp32", device=None, filter="fft",
                 keep_projections=False, parker=False):
        if geom is None:
            raise ValueError("geometry is required")
        if store not in _STORE_DTYPES:
            raise ValueError(f"unknown store {store!r}: use one of {sorted(_STORE_DTYPES)}")
        if filter not in ("fft", "tc", "tc-bf16"):
            raise ValueError(f"unknown filter {filter!r}: use 'fft', 'tc' or 'tc-bf16'")
        if filter != "fft" and geom.cols > 512:
            raise ValueError("the tensor-core filter supports detector rows of at most 512 columns")
        self.filter_method = filter
        self.device = _device(device)
        N.load()
        self.requested_backend = backend
        self.backend = BACKEND
        self.geom = geom
        self.window = window
        self.gaussian = float(gaussian)
        self.tilt = float(tilt)
        self.verbose = verbose
        self.store = store
        self.box = np.asarray(geom.volume_box(), dtype=float)
        self.n_total = geom.n_angles
        self.cor_shift = 0.0
        self.version = 0
        self._lock = threading.RLock()
        self._ingest_lock = threading.Lock()
        self._order = np.zeros(self.n_total, dtype=np.int64)
        self._received = np.zeros(self.n_total, dtype=bool)
        self.n = 0
        R, C = geom.rows, geom.cols
        self._dtype_code, tdtype = _STORE_DTYPES[store]
        self._pitch = ring_pitch(C, store)

        if isinstance(geom, ParallelGeometry):
            self.kind = "parallel"
            self._kind_code = N.MR_PARALLEL
            self._band_axis = (0.0, 0.0, 1.0)      # detector rows follow z
            self._maps_all = parallel_view_maps(geom.angles, geom.pixel_u, geom.pixel_v, R, C)
        elif isinstance(geom, ConeVecGeometry):
            self.kind = "cone"
            self._kind_code = N.MR_CONE
            self._K_all = cone_constants(geom.vectors)
            self._maps_all = cone_view_maps(self._K_all, R, C)
            # the orbit's axis as the mean detector row direction (tile order only)
            vm = np.asarray(geom.vectors, dtype=np.float64)[:, 9:12]
            vm = (vm / np.linalg.norm(vm, axis=1, keepdims=True)).mean(0)
            nrm = float(np.linalg.norm(vm))
            self._band_axis = tuple(vm / nrm) if nrm > 1e-6 else None
            if geom.angular_range < 2 * np.pi - 1e-3 and verbose and not parker:
                print("note: short scan (<360 deg) - no Parker weights, expect some artefacts")
        else:
            raise TypeError(type(geom))
        ramp_response(C, 1.0, window)          # validates the window name early

        with torch.cuda.device(self.device):
            self.stream = torch.cuda.Stream(self.device)          # reconstruction
            self.ingest_stream = torch.cuda.Stream(self.device)   # filtering of new views
            self.copy_stream = torch.cuda.Stream(self.device)     # host -> device raw counts
            self._tables = _FilterTables(C, window, self.device)
            # per-view constants of the whole orbit, computed once: the filter records
            # (slot filled in per call) and a device copy of the view records
            if self.kind == "cone":
                self._fv_all = cone_filter_views(self._K_all, R, C, self._tables.n_fft, 0)
            else:
                self._fv_all = parallel_filter_views(geom.pixel_u, self.n_total, self._tables.n_fft, 0)
            self._maps_dev = torch.from_numpy(self._maps_all.view(np.uint8).copy()).to(self.device)
            _staging(self.device)               # page-locked record staging, taken up front
            self._ring = torch.zeros((self.n_total, R, self._pitch), dtype=tdtype, device=self.device)
            self._views_host = np.zeros(self.n_total, dtype=N.VIEW_DTYPE)
            self._views_dev = torch.zeros(self.n_total * N.VIEW_DTYPE.itemsize, dtype=torch.uint8,
                                          device=self.device)
        self._ring_c = _ring_struct(self._ring, self._dtype_code, self._kind_code, R, C)
        self._parker = None             # [n_total, C] f32 short-scan weights (device)
        if parker:
            if self.kind != "cone":
                raise ValueError("Parker weights apply to cone-beam orbits")
            with torch.cuda.device(self.device):
                pw = parker_weights(geom.vectors, C)
                self._parker = torch.from_numpy(pw.astype(np.float32)).to(self.device)
            # views weighted by the plateau value in every column (most of the orbit)
            self._parker_plateau = float(pw.max())
            self._parker_flat = np.all(pw == pw.max(), axis=1)
        self._proj = None               # unfiltered line integrals [n_total, R, pitch] (keep_projections)
        if keep_projections:
            with torch.cuda.device(self.device):
                self._proj = torch.zeros((self.n_total, R, self._pitch), dtype=torch.float32, device=self.device)
        self._ingest_event = None
        # (slot_end, event) of the chunks of the latest host upload: a reconstruction can
        # sum the views of each chunk as soon as that chunk is filtered
        self._chunk_marks = []
        self._raw_dev = None            # device staging of host raw counts (grows on demand)
        self._raw_pinned = []           # pinned staging of pageable raw counts, one per chunk slot
        self.upload_chunk_bytes = 16 << 20   # raw bytes per overlapped upload + ingest chunk
        self.upload_middle_chunks = 4        # page-locked sources: inner chunks this many times larger
        self.kernel_timer = None        # a KernelTimer records launch durations when set
        self.bp_kernel = "staged"       # "plain": direct-gather kernel for every request
        with torch.cuda.device(self.device):
            self._status = torch.zeros(1, dtype=torch.int32, device=self.device)

        if proj is not None:
            t0 = time.perf_counter()
            for i in range(0, self.n_total, 64):
                self.add_projections(np.arange(i, min(i + 64, self.n_total)), proj[:, i:i + 64, :])
            if verbose:
                torch.cuda.synchronize(self.device)
                print(f"[minirecast] filtered {self.n} projections ({geom.rows}x{geom.cols}) "
                      f"in {time.perf_counter() - t0:.2f}s, backend={self.backend}")

    # ----------------------------------------------------------- ingest
    def _filter_views(self, idx, slots):
        """mr_filter_view records of geometry views `idx` bound for ring `slots`."""
        fv = self._fv_all[idx]
        fv["slot"] = slots
        return fv

    @staticmethod
    def _first_of_run(indices):
        """indices[0] when `indices` are consecutive ascending view numbers, else None."""
        i0 = int(indices[0])
        if int(indices[-1]) - i0 == len(indices) - 1 and (len(indices) < 3 or (np.diff(indices) == 1).all()):
            return i0
        return None

    def _upload_view_records(self, indices, slots):
        """Queue the mr_view records of new slots on the ingest stream (asynchronous). This
        is the only writer of the device table and keeps `_views_host` as its mirror, so
        slots that already hold the same records - a new scan of the same orbit in the same
        order after reset() - need no copy. Called under the ingest lock."""
        n0, n1 = slots[0], slots[-1] + 1
        sz = N.VIEW_DTYPE.itemsize
        i0 = self._first_of_run(indices)
        new = self._maps_all[i0:i0 + n1 - n0] if i0 is not None else self._maps_all[indices]
        if new.tobytes() == self._views_host[n0:n1].tobytes():
            return
        self._views_host[n0:n1] = new
        with torch.cuda.stream(self.ingest_stream):
            dst = self._views_dev[n0 * sz:n1 * sz]
            if i0 is not None:
                # a run of consecutive views: a device-to-device copy of the orbit's records
                dst.copy_(self._maps_dev[i0 * sz:(i0 + n1 - n0) * sz], non_blocking=True)
                return
            # page-locked staging: the copy is asynchronous and the host does not wait for
            # the ingest kernels queued before it
            recs = np.ascontiguousarray(self._maps_all[indices]).view(np.uint8).reshape(-1)
            if _staging(self.device).upload(recs, self.device, out=dst) is None:
                dst.copy_(torch.from_numpy(recs.copy()).pin_memory(), non_blocking=True)

    def _admit(self, indices, slots, event, uploaded=False, marks=()):
        """Make filtered slots visible to reconstructions (under the state lock)."""
        with self._lock:
            n0, n1 = slots[0], slots[-1] + 1
            self._order[n0:n1] = indices
            self._received[indices] = True
            if not uploaded:
                self._upload_view_records(indices, slots)
            self._chunk_marks = list(marks)
            event.record(self.ingest_stream)
            self._ingest_event = event
            self.n = int(n1)
            self.version += 1
            return self.n

    def add_projections(self, indices, block):
        """Add projections (geometry indices `indices`, data [rows, k, cols] float32)."""
        return self._add_block(indices, block)

    def _add_block(self, indices, block, x_bound=None):
        """add_projections; x_bound: a known bound on |block| (see filter_block_device)."""
        indices = np.asarray(indices, dtype=np.int64).ravel()
        is_tensor = isinstance(block, torch.Tensor)
        if not is_tensor:
            block = np.asarray(block, dtype=np.float32)
        if block.shape[1] != len(indices):
            raise ValueError("block has %d projections but %d indices"
                             % (block.shape[1], len(indices)))
        with self._ingest_lock:
            keep = ~self._received[indices]
            if not keep.all():
                indices = indices[keep]
                block = block[:, torch.from_numpy(keep)] if is_tensor else block[:, keep, :]
            if len(indices) == 0:
                return self.n
            k = len(indices)
            R, C = self.geom.rows, self.geom.cols
            n0 = self.n
            slots = np.arange(n0, n0 + k)
            with torch.cuda.device(self.device), torch.cuda.stream(self.ingest_stream):
                x = _to_device_tensor(block, self.device, torch.float32)      # [R, k, C]
                x, s_view, s_row = preprocess.apply_device(x, self.gaussian, self.tilt)
                if self._proj is not None:
                    self._proj[n0:n0 + k, :, :C] = torch.as_strided(x, (k, R, C), (s_view, s_row, 1))
                if self._parker is not None:
                    # short-scan weights on a copy (x may be the caller's own tensor)
                    idx_dev = _struct_tensor(indices, self.device, asynchronous=True).view(torch.int64)
                    w = self._parker.index_select(0, idx_dev)                            # [k, C]
                    xw = torch.empty((k, R, C), dtype=torch.float32, device=self.device)
                    torch.mul(torch.as_strided(x, (k, R, C), (s_view, s_row, 1)), w[:, None, :], out=xw)
                    x, s_view, s_row = xw, R * C, C
                fv = _struct_tensor(self._filter_views(indices, slots), self.device)
                filter_block_device(x, s_view, s_row, k, fv, self._tables, self._ring_c,
                                    self.ingest_stream, self.filter_method, self._status,
                                    None if x_bound is None else x_bound * (self._parker_plateau
                                                                            if self._parker is not None else 1.0))
                ev = torch.cuda.Event()
            return self._admit(indices, slots, ev)

    def reset(self):
        """Forget every received view (a new scan with the same geometry); the device
        ring is reused."""
        with self._ingest_lock, self._lock:
            # new views may overwrite slots only after queued reconstructions read them
            ev = torch.cuda.Event()
            ev.record(self.stream)
            self.ingest_stream.wait_event(ev)
            self._received[:] = False
            self._chunk_marks = []
            self.n = 0
            self.version += 1

    def set_flat_dark(self, flat, dark, bin=1, flip_rows=False, mode="flexray"):
        """Flat / dark frames ([n, R0, C0] or [R0, C0], uint16 or float) for
        add_raw_projections, prepared like the reference loaders: mean binning of each
        frame, row flip (FleX-ray, flexray.py:111-116), mean over frames, then
        gain = 1/max(F-D, 1) ("flexray", flexray.py:174-177) or 1/max(F-D, 1e-6)
        ("hdf5", hdf5.py:64-77). Binned size must equal the geometry's rows x cols."""
        if mode not in ("flexray", "hdf5"):
            raise ValueError(f"unknown mode {mode!r}")
        R, C = self.geom.rows, self.geom.cols
        b = int(bin)

        def binned(frames):
            t = torch.as_tensor(np.asarray(frames, dtype=np.float32)).to(self.device)
            if t.ndim == 2:
                t = t[None]
            h, w = t.shape[1] // b * b, t.shape[2] // b * b
            t = t[:, :h, :w].reshape(t.shape[0], h // b, b, w // b, b).mean(dim=(2, 4))
            if flip_rows:
                t = torch.flip(t, dims=[1])
            return t.mean(0)

        with torch.cuda.device(self.device), torch.cuda.stream(self.ingest_stream):
            d = binned(dark)
            f = binned(flat)
            if tuple(d.shape) != (R, C):
                raise ValueError(f"binned frames are {tuple(d.shape)}, geometry is {(R, C)}")
            eps = 1.0 if mode == "flexray" else 1e-6
            self._dark = d.contiguous()
            self._gain = (1.0 / torch.clamp(f - d, min=eps)).contiguous()
        self._raw_bin, self._raw_flip = b, bool(flip_rows)

    def add_raw_projections(self, indices, raw):
        """Fused ingest of raw detector counts: raw [k, R0, C0] uint16 (NumPy, pinned or
        CUDA tensor) -> bin, (P-D)*gain, clip 1e-3, -log, FDK weight, ramp filter, store
        (mr_ingest_u16). A CUDA tensor is filtered in one launch; host counts are uploaded
        in chunks whose transfers overlap the filtering of the previous chunk. Needs
        set_flat_dark() first."""
        if getattr(self, "_gain", None) is None:
            raise RuntimeError("call set_flat_dark() before add_raw_projections()")
        if self.gaussian or self.tilt:
            raise ValueError("gaussian / tilt pre-processing needs add_projections() "
                             "(the fused raw ingest has no neighbourhood pass)")
        indices = np.asarray(indices, dtype=np.int64).ravel()
        if raw.shape[0] != len(indices):
            raise ValueError("raw has %d projections but %d indices" % (raw.shape[0], len(indices)))
        b = self._raw_bin
        R, C = self.geom.rows, self.geom.cols
        if raw.shape[1] < R * b or raw.shape[2] < C * b:
            raise ValueError(f"raw frames {tuple(raw.shape[1:])} are smaller than "
                             f"{R * b} x {C * b}")
        if self._parker is not None:
            return self._add_raw_parker(indices, raw)
        return self._add_raw_fused(indices, raw)

    def _add_raw_parker(self, indices, raw):
        """Short scan: a view whose Parker weight is the plateau value for every column
        (the middle of the orbit) goes through the fused ingest with that value folded into
        the filter's output scale (the filter is linear); the others are corrected on their
        own (mr_correct_u16), weighted per column and filtered as a block."""
        const = self._parker_flat[indices]
        if const.all():
            return self._add_raw_fused(indices, raw, self._parker_plateau)
        if not const.any():
            return self._add_block(indices, self._correct_raw(raw), RAW_LINE_BOUND)
        flat, ramp = np.flatnonzero(const), np.flatnonzero(~const)
        self._add_raw_fused(indices[flat], self._views_of(raw, flat), self._parker_plateau)
        return self._add_block(indices[ramp], self._correct_raw(self._views_of(raw, ramp)), RAW_LINE_BOUND)

    @staticmethod
    def _views_of(raw, sel):
        """raw[sel] for raw counts [k, R0, C0] (a view when sel is a run)."""
        if len(sel) and int(sel[-1]) - int(sel[0]) == len(sel) - 1:
            return raw[int(sel[0]):int(sel[-1]) + 1]
        if isinstance(raw, torch.Tensor):
            return raw[torch.from_numpy(sel).to(raw.device)]
        return np.asarray(raw)[sel]

    def _add_raw_fused(self, indices, raw, out_scale=1.0):
        """The fused ingest of add_raw_projections; out_scale multiplies the filtered views."""
        with self._ingest_lock:
            keep = ~self._received[indices]
            if not keep.all():
                indices = indices[keep]
                raw = raw[torch.from_numpy(keep)] if isinstance(raw, torch.Tensor) else raw[keep]
            if len(indices) == 0:
                return self.n
            k = len(indices)
            n0 = self.n
            slots = np.arange(n0, n0 + k)
            on_device = isinstance(raw, torch.Tensor) and raw.is_cuda
            if self._proj is not None:
                self._keep_raw_line_integrals(raw, n0, k)

            def prepare():
                # filter records of the new slots and their view records, queued on the
                # ingest stream ahead of the first ingest launch (the view records go
                # before any chunk is filtered, so a reconstruction may use the first
                # chunks of this call while the later ones are still on the bus)
                fv_host = self._filter_views(indices, slots)
                if out_scale != 1.0:
                    fv_host["out_scale"] *= out_scale
                # the filter records go up on the copy stream: unlike the view records they
                # do not wait for the reconstructions that still read the ring
                with torch.cuda.stream(self.copy_stream):
                    fv = _struct_tensor(fv_host, self.device, asynchronous=True)
                    fv_ready = torch.cuda.Event()
                    fv_ready.record(self.copy_stream)
                self.ingest_stream.wait_event(fv_ready)
                fv.record_stream(self.ingest_stream)
                self._upload_view_records(indices, slots)
                return fv

            marks = []
            with torch.cuda.device(self.device), torch.cuda.stream(self.ingest_stream):
                if on_device:
                    x = raw.view(torch.int16) if raw.dtype == torch.uint16 else raw
                    x = x.to(self.device, non_blocking=True).contiguous()
                    if x.element_size() != 2:
                        raise ValueError("raw counts must be 16-bit")
                    self._ingest_launch(x, 0, k, prepare())
                    x.record_stream(self.ingest_stream)
                else:
                    marks = [(n0 + c1, e) for c1, e in self._ingest_host(raw, k, prepare)[:-1]]
                ev = torch.cuda.Event()
            return self._admit(indices, slots, ev, uploaded=True, marks=marks)

    def _correct_raw(self, raw):
        """Line integrals [rows, k, cols] f32 (device) of raw counts [k, R0, C0]: the
        correction of the fused ingest (bin, row flip, (P-D)*gain, clip, -log) alone."""
        R, C, b = self.geom.rows, self.geom.cols, self._raw_bin
        with torch.cuda.device(self.device), torch.cuda.stream(self.ingest_stream):
            if isinstance(raw, torch.Tensor):
                t = raw.view(torch.int16) if raw.dtype == torch.uint16 else raw
                if t.element_size() != 2:
                    raise ValueError("raw counts must be 16-bit")
            else:
                arr = np.asarray(raw)
                if arr.dtype.itemsize != 2:
                    raise ValueError("raw counts must be 16-bit")
                t = torch.from_numpy(np.ascontiguousarray(arr).view(np.int16))
            t = t.to(self.device, non_blocking=True).contiguous()
            k, R0, C0 = t.shape
            out = torch.empty((R, k, C), dtype=torch.float32, device=self.device)
            for v0 in range(0, k, 65535):
                v1 = min(k, v0 + 65535)
                N.check(N.load().mr_correct_u16(ctypes_void(t[v0].data_ptr()), R0 * C0, C0, v1 - v0, b,
                                                int(self._raw_flip), R, 0, 0, R, C, ctypes_void(self._dark.data_ptr()),
                                                ctypes_void(self._gain.data_ptr()), C, N.MR_CORRECT_FLEXRAY,
                                                ctypes_void(out[:, v0].data_ptr()), k * C, C,
                                                ctypes_void(self.ingest_stream.cuda_stream)), "mr_correct_u16")
            t.record_stream(self.ingest_stream)
        return out

    def _keep_raw_line_integrals(self, raw, n0, k):
        """-log(max((binned counts - dark) * gain, 1e-3)) of k raw views into the kept
        projections (the correction of the fused ingest, without its filter)."""
        b, R, C = self._raw_bin, self.geom.rows, self.geom.cols
        with torch.cuda.device(self.device), torch.cuda.stream(self.ingest_stream):
            t = raw if isinstance(raw, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(raw).view(np.int16))
            t = t.to(self.device, non_blocking=True)
            t = (t.view(torch.int16).to(torch.int32) & 0xFFFF).to(torch.float32)       # uint16 counts
            t = t[:, :R * b, :C * b].reshape(k, R, b, C, b).mean(dim=(2, 4))
            if self._raw_flip:
                t = torch.flip(t, dims=[1])
            x = -torch.log(torch.clamp((t - self._dark) * self._gain, min=1e-3))
            self._proj[n0:n0 + k, :, :C] = x

    def refine_slice_ls(self, origin=(0.0, 0.0, 0.0), normal=(0.0, 0.0, 1.0), n=256, size=None, zoom=1.0,
                        center=None, iters=10):
        """Least-squares refinement of a slice from the views received so far (few views
        during a live scan): CGLS on min ||A x - c p||^2 over the slice's in-box samples,
        started from the FBP slice. A is the matched forward projector of the slice
        samples (the exact transpose of the bilinear back-projection, mr_project_adjoint),
        A^T the plain back-projection, p the kept unfiltered line integrals
        (keep_projections=True), c the least-squares scale that makes the FBP slice x0 fit
        A x0 ~ c p (the sample-spacing factor of the discretisation).
        The slice is modelled as the only object on its rays, which is exact for axial
        slices of a parallel-beam scan placed on a detector row (each detector row sees one
        axial slice) and an approximation otherwise (cone beam near the mid-plane).
        Returns (img [n, n] f64, residual norms per iteration)."""
        from .autograd import BackprojectOp
        if self._proj is None:
            raise RuntimeError("refine_slice_ls needs SliceReconstructor(..., keep_projections=True)")
        n_views, shift, ev = self._snapshot()
        if n_views == 0:
            raise RuntimeError("no projections received yet")
        grid = plane_grid(self.box, origin, normal, int(n), size, zoom, center, shift)
        grids = np.zeros(1, dtype=N.GRID_DTYPE)
        grids[0] = grid
        R, C = self.geom.rows, self.geom.cols
        with torch.cuda.device(self.device), torch.cuda.stream(self.stream):
            if ev is not None:
                self.stream.wait_event(ev)
            op = BackprojectOp(self._views_dev, self._kind_code, R, C, grids, n * n, n_views, scale=1.0)
            fbp = BackprojectOp(self._views_dev, self._kind_code, R, C, grids, n * n, n_views)
            x = fbp.forward(self._ring, shift)
            shape = (n_views, R, self._pitch)
            # detector pixels the slice reaches with a real weight (FP32 coordinates can put
            # ~1e-6 of a sample on a neighbouring row): the data term covers only those
            w1 = op.adjoint(torch.ones(n * n, dtype=torch.float32, device=self.device), shift, 0.0, shape)
            mask = (w1 > 1e-3 * float(w1.max())).float()
            A = lambda v: op.adjoint(v, shift, 0.0, shape) * mask         # noqa: E731  samples -> detector
            AT = lambda r: op.forward(r * mask, shift)                    # noqa: E731  detector -> samples
            p = self._proj[:n_views]
            Ax = A(x)
            pm = p * mask
            c = float((Ax * pm).sum() / (pm * pm).sum().clamp_min(1e-30))
            b = c * pm
            r = b - Ax
            s = AT(r)
            d = s.clone()
            gamma = float((s * s).sum())
            hist = [float(r.norm())]
            for _ in range(int(iters)):
                if gamma <= 0.0:
                    break
                q = A(d)
                qq = float((q * q).sum())
                if qq <= 0.0:
                    break
                alpha = gamma / qq
                x = x + alpha * d
                r = r - alpha * q
                s = AT(r)
                gamma_new = float((s * s).sum())
                d = s + (gamma_new / gamma) * d
                gamma = gamma_new
                hist.append(float(r.norm()))
            img = x.view(n, n).double().cpu().numpy()
        return img, hist

    def _ingest_launch(self, x, c0, c1, fv, stream=None):
        """mr_ingest_u16 of views [c0, c1) of the device raw block x on `stream` (default:
        the ingest stream)."""
        lib = N.load()
        t = self._tables
        tm = self.kernel_timer
        stream = self.ingest_stream if stream is None else stream
        name = "mr_ingest_u16" if self.filter_method == "fft" else "mr_ingest_u16_tc"
        ev0 = tm.start(stream) if tm is not None else None
        view_bytes = x.shape[1] * x.shape[2] * 2
        common = (ctypes_void(x.data_ptr() + c0 * view_bytes), x.shape[1] * x.shape[2], x.shape[2],
                  self._raw_bin, int(self._raw_flip), ctypes_void(self._dark.data_ptr()),
                  ctypes_void(self._gain.data_ptr()), c1 - c0,
                  ctypes_void(fv.data_ptr() + c0 * N.FILTER_VIEW_DTYPE.itemsize))
        if self.filter_method == "fft":
            st = lib.mr_ingest_u16(*common, ctypes_void(t.H.data_ptr()), ctypes_void(t.tw.data_ptr()), t.log2n,
                                   self._ring_c, ctypes_void(stream.cuda_stream))
        else:
            fmt = N.MR_BF16 if self.filter_method == "tc-bf16" else N.MR_F16
            img, t_scale = t.tc_image(fmt)
            st = lib.mr_ingest_u16_tc(*common, ctypes_void(img.data_ptr()), fmt, t_scale, t.n_fft, self._ring_c,
                                      ctypes_void(self._status.data_ptr()), ctypes_void(stream.cuda_stream))
        if tm is not None:
            tm.stop(name, ev0, stream)
        N.check(st, name)

    def _ingest_host(self, raw, k, prepare):
        """Upload host raw counts in chunks on the copy stream and filter each chunk on the
        ingest stream as soon as it has landed, so the PCIe transfer of chunk i+1 overlaps
        the ingest of chunk i. Pinned torch tensors are copied directly; anything else
        (NumPy, pageable tensors) is staged through reusable pinned buffers. `prepare()`
        (host-side records of the new views, returning the device filter records) runs
        once the first chunk is on the bus, so the transfer does not wait for it.
        Returns [(views done, event)] per chunk."""
        if isinstance(raw, torch.Tensor):
            if raw.element_size() != 2:
                raise ValueError("raw counts must be 16-bit")
            host = raw.view(torch.int16) if raw.dtype == torch.uint16 else raw
            host = host.contiguous()
            pinned = host.is_pinned()
            host_np = None if pinned else host.numpy()
        else:
            arr = np.asarray(raw)
            if arr.dtype.itemsize != 2:
                raise ValueError("raw counts must be 16-bit")
            host_np = np.ascontiguousarray(arr).view(np.int16)
            host, pinned = None, False
        shape = tuple(host.shape if host is not None else host_np.shape)
        view_bytes = shape[1] * shape[2] * 2
        chunk = max(1, min(k, self.upload_chunk_bytes // view_bytes))
        need = k * shape[1] * shape[2]
        if self._raw_dev is None or self._raw_dev.numel() < need:
            self._raw_dev = torch.empty(need, dtype=torch.int16, device=self.device)
        x = self._raw_dev[:need].view(k, shape[1], shape[2])
        # the previous call's ingest kernels must be done reading the staging buffer
        self.copy_stream.wait_stream(self.ingest_stream)
        marks = []                      # (views done, event) per chunk
        if not pinned:
            n_slots = 3
            while len(self._raw_pinned) < n_slots:
                self._raw_pinned.append([None, None])        # [pinned tensor, event of its last copy]
        if pinned and self.upload_middle_chunks > 1 and k > 4 * chunk:
            # the first chunk and the last two keep their size (the ingest starts early, and
            # the filtering and summing of a large chunk is done before the last one lands,
            # so little work is left after the transfer); the ones between are larger, so the
            # transfer is cut into fewer copies
            inner = k - 3 * chunk
            n_in = -(-inner // (chunk * self.upload_middle_chunks))
            cuts = [chunk + (inner * j) // n_in for j in range(n_in + 1)]
            bounds = [0] + cuts + [k - chunk, k]
        else:
            bounds = list(range(0, k, chunk)) + [k]
        for i, (c0, c1) in enumerate(zip(bounds[:-1], bounds[1:])):
            with torch.cuda.stream(self.copy_stream):
                if pinned:
                    x[c0:c1].copy_(host[c0:c1], non_blocking=True)
                else:
                    slot = self._raw_pinned[i % len(self._raw_pinned)]
                    n_el = (c1 - c0) * shape[1] * shape[2]
                    if slot[0] is None or slot[0].numel() < chunk * shape[1] * shape[2]:
                        slot[0] = torch.empty(chunk * shape[1] * shape[2], dtype=torch.int16).pin_memory()
                    elif slot[1] is not None:
                        slot[1].synchronize()                # its previous copy has left the buffer
                    buf = slot[0][:n_el]
                    np.copyto(buf.numpy(), host_np[c0:c1].reshape(-1))
                    x[c0:c1].copy_(buf.view(c1 - c0, shape[1], shape[2]), non_blocking=True)
                    slot[1] = torch.cuda.Event()
                    slot[1].record(self.copy_stream)
                landed = torch.cuda.Event()
                landed.record(self.copy_stream)
            if i == 0:
                fv = prepare()
            self.ingest_stream.wait_event(landed)
            self._ingest_launch(x, c0, c1, fv)
            done = torch.cuda.Event()
            done.record(self.ingest_stream)
            marks.append((c1, done))
        return marks

    # ----------------------------------------------------------- info
    @property
    def native_pixel(self):
        """Detector pixel size at the rotation axis (mm)."""
        if self.kind == "parallel":
            return float(self.geom.pixel_u)
        K = self._K_all
        return float(np.linalg.norm(K["u"][0]) * K["sod"][0] / K["sdd"][0])

    def info(self):
        return dict(kind=self.kind, n=int(self.n), n_total=int(self.n_total),
                    version=int(self.version), cor_shift=float(self.cor_shift),
                    box=[float(b) for b in self.box], native_pixel=self.native_pixel,
                    backend=self.backend)

    def plane_size(self, normal):
        return plane_size_for_box(self.box, normal)

    def inside_box(self, pts):
        return np.all(np.abs(pts) <= self.box, axis=-1)

    # ----------------------------------------------------------- reconstruction
    def _snapshot(self):
        with self._lock:
            return self.n, self.cor_shift, self._ingest_event

    def _run_grids(self, grids, out, n, event):
        """Launch the batched back-projection of `grids` into device `out`. Right after a
        chunked host upload, the views are summed chunk by chunk: each partial launch
        waits only for its own chunk's filter, so the reconstruction overlaps the transfer
        of the later chunks (same scale; FP32 partial sums added in view order)."""
        stream = self.stream
        grids["scale"] = np.pi / n if n else 0.0
        marks = [(se, e) for se, e in self._chunk_marks if 0 < se < n]
        regular = not (np.asarray(grids["flags"]) & N.MR_GRID_POINTS).any()
        if marks and regular and self.bp_kernel == "staged":
            bounds = [0] + [se for se, _ in marks] + [n]
            events = [e for _, e in marks] + [event]
            G = len(grids)
            parts = np.tile(np.ascontiguousarray(grids, dtype=N.GRID_DTYPE), len(events))
            for i, (a, b) in enumerate(zip(bounds[:-1], bounds[1:])):
                sl = slice(i * G, (i + 1) * G)
                parts["view_begin"][sl], parts["n_views"][sl] = a, b - a
                parts["accumulate"][sl] = 0 if i == 0 else 1
            tiles = N.plan_tiles(grids, self._band_axis)     # the same tiles for every view range
            if len(tiles) == 0:
                return
            lib = N.load()
            v = ctypes_void
            with torch.cuda.device(self.device), torch.cuda.stream(stream):
                # one upload for all ranges and the tiles; launch i reads its own G records
                recs = _struct_tensor(np.concatenate([parts.view(np.uint8), tiles.view(np.uint8)]), self.device)
                g_ptr, t_ptr = recs.data_ptr(), recs.data_ptr() + parts.nbytes
                st_ptr = v(self._status.data_ptr())
                for i, ((a, b), e) in enumerate(zip(zip(bounds[:-1], bounds[1:]), events)):
                    if e is not None:
                        stream.wait_event(e)
                    tm = self.kernel_timer
                    ev0 = tm.start(stream) if tm is not None else None
                    rc = lib.mr_backproject_staged(self._ring_c, v(self._views_dev.data_ptr()),
                                                   v(g_ptr + i * G * N.GRID_DTYPE.itemsize),
                                                   v(t_ptr), len(tiles), v(out.data_ptr()), st_ptr,
                                                   v(stream.cuda_stream))
                    if tm is not None:
                        tm.stop("mr_backproject_staged", ev0, stream)
                    N.check(rc, "mr_backproject_staged")
                recs.record_stream(stream)
            return
        grids["n_views"] = n
        with torch.cuda.device(self.device), torch.cuda.stream(stream):
            # no chunked host upload in flight (it would sit ahead of a page-locked copy on
            # the copy engines): the records go up without the host waiting
            backproject_device(self._ring_c, self._views_dev, grids, out, stream, self.device,
                               self.kernel_timer, self.bp_kernel, self._status, wait=event,
                               asynchronous=not self._chunk_marks, band_axis=self._band_axis)

    def reconstruct_points_tensor(self, pts, cor_shift=None):
        """Device variant of reconstruct_points: pts (M, 3) -> f32 tensor [M]."""
        n, shift, ev = self._snapshot()
        if cor_shift is not None:
            shift = float(cor_shift)
        with torch.cuda.device(self.device), torch.cuda.stream(self.stream):
            p = _to_device_tensor(pts, self.device, torch.float32).reshape(-1, 3).contiguous()
            M = p.shape[0]
            out = torch.zeros(M, dtype=torch.float32, device=self.device)
            if n == 0 or M == 0:
                return out
            g = np.zeros(1, dtype=N.GRID_DTYPE)
            g["n_i"], g["n_j"], g["n_k"] = 1, M, 1
            g["flags"] = N.MR_GRID_POINTS
            g["out_stride_j"] = 1
            g["points"] = p.data_ptr()
            g["cor_shift"] = shift
            self._run_grids(g, out, n, ev)
            p.record_stream(self.stream)
        _handoff(self.stream, out)
        return out

    def reconstruct_points(self, pts, cor_shift=None):
        pts = np.ascontiguousarray(np.asarray(pts, dtype=np.float64).reshape(-1, 3))
        out = self.reconstruct_points_tensor(pts, cor_shift)
        return out.cpu().numpy().astype(np.float64)

    def plane_grid(self, origin, normal, n=256, size=None, zoom=1.0, center=None, cor_shift=None):
        shift = self.cor_shift if cor_shift is None else float(cor_shift)
        return plane_grid(self.box, origin, normal, int(n), size, zoom, center, shift)

    def _plane_record(self, origin, normal, n, size, zoom, center, shift):
        """plane_grid for this reconstructor's box, memoised on the request's parameters
        (the FP64 plane set-up is pure; a repeated request skips it on the host)."""
        flat = lambda v: None if v is None else tuple(float(x) for x in np.ravel(v))   # noqa: E731
        key = (flat(origin), flat(normal), int(n), None if size is None else float(size), float(zoom),
               flat(center), float(shift))
        cache = self.__dict__.setdefault("_plane_cache", collections.OrderedDict())
        rec = cache.get(key)
        if rec is None:
            rec = plane_grid(self.box, origin, normal, n, size, zoom, center, shift)
            cache[key] = rec
            if len(cache) > 256:
                cache.popitem(last=False)
        else:
            cache.move_to_end(key)
        return rec.copy()

    def _planes(self, requests):
        """One batched launch for many slices -> (flat f32 device tensor, sizes)."""
        n_views, shift, ev = self._snapshot()
        grids = np.zeros(len(requests), dtype=N.GRID_DTYPE)
        sizes, offset = [], 0
        for r, req in enumerate(requests):
            n = int(req.get("n", 256))
            s_ = req.get("cor_shift")
            grids[r] = self._plane_record(req["origin"], req["normal"], n, req.get("size"),
                                          req.get("zoom", 1.0), req.get("center"),
                                          shift if s_ is None else float(s_))
            grids[r]["out_offset"] = offset
            sizes.append(n)
            offset += n * n
        with torch.cuda.device(self.device), torch.cuda.stream(self.stream):
            out = torch.zeros(offset, dtype=torch.float32, device=self.device)
            if n_views > 0 and offset > 0:
                self._run_grids(grids, out, n_views, ev)
        _handoff(self.stream, out)
        return out, sizes

    def reconstruct_planes_tensor(self, requests):
        """Back-project many slices in ONE launch. `requests` is a list of dicts with
        the reconstruct_plane arguments (origin, normal, n, size, zoom, center,
        cor_shift). Returns a list of f32 device tensors [n, n] (views of one buffer)."""
        out, sizes = self._planes(requests)
        res, o = [], 0
        for n in sizes:
            res.append(out[o:o + n * n].view(n, n))
            o += n * n
        return res

    def reconstruct_planes(self, requests):
        """Batched reconstruct_plane without the point arrays: list of f64 images
        (one device->host copy for the whole batch). The images are widened to f64 on the
        device and copied into one pinned host buffer, which the returned arrays view
        (the pinned block goes back to torch's host cache when they are freed)."""
        out, sizes = self._planes(requests)
        pinned = torch.empty(out.shape, dtype=torch.float64, pin_memory=True)
        with torch.cuda.device(self.device), torch.cuda.stream(self.stream):
            wide = out.to(torch.float64)
            pinned.copy_(wide, non_blocking=True)
        self.stream.synchronize()
        host = pinned.numpy()
        res, o = [], 0
        for n in sizes:
            res.append(host[o:o + n * n].reshape(n, n))
            o += n * n
        return res

    def reconstruct_plane(self, origin, normal, n=256, size=None, zoom=1.0, center=None,
                          cor_shift=None):
        """Reconstruct an n x n slice of the plane through `origin` with the given normal.
        Returns (image [n, n] float64, points [n, n, 3]); pixels outside the box are 0."""
        img = self.reconstruct_planes([dict(origin=origin, normal=normal, n=n, size=size,
                                            zoom=zoom, center=center, cor_shift=cor_shift)])[0]
        pts, _ = slice_points(self.box, origin, normal, n, size, zoom, center)
        return img, pts

    def _volume_frame(self, voxel, maxdim):
        if maxdim is not None:
            dims, origin, h = volume_grid(self.box, maxdim)
        else:
            h = float(voxel or self.native_pixel)
            dims = np.maximum(np.ceil(2.0 * self.box / h).astype(int), 2)
            origin = -self.box + h / 2.0
        return tuple(int(d) for d in dims), np.asarray(origin, float), h

    def reconstruct_volume_tensor(self, voxel=None, maxdim=None, chunk=None, progress=None,
                                  out=None):
        """Device variant of reconstruct_volume: returns (f32 tensor [nx, ny, nz], origin, h)."""
        dims, origin, h = self._volume_frame(voxel, maxdim)
        nx, ny, nz = dims
        n_views, shift, ev = self._snapshot()
        with torch.cuda.device(self.device), torch.cuda.stream(self.stream):
            vol = out if out is not None else torch.empty((nx, ny, nz), dtype=torch.float32,
                                                          device=self.device)
            if n_views == 0:
                vol.zero_()
                return vol, origin, h
            planes = nx if chunk is None else max(1, int(chunk) // (ny * nz))
            for k0 in range(0, nx, planes):
                k1 = min(nx, k0 + planes)
                g = np.zeros(1, dtype=N.GRID_DTYPE)
                g[0] = volume_grid_record(origin, h, dims, k0, k1)
                g["cor_shift"] = shift
                self._run_grids(g, vol.view(-1), n_views, ev)
                if progress is not None:
                    self.stream.synchronize()
                    progress((k1 - 1) / max(nx - 1, 1))
        _handoff(self.stream, vol)
        return vol, origin, h

    def reconstruct_volume_slab_tensor(self, k0, k1, voxel=None, maxdim=None):
        """x-planes [k0, k1) of the volume of reconstruct_volume (same frame), as a device
        tensor [k1 - k0, ny, nz]: the unit of work of a volume sharded over GPUs."""
        dims, origin, h = self._volume_frame(voxel, maxdim)
        nx, ny, nz = dims
        k0, k1 = int(k0), int(k1)
        if not 0 <= k0 <= k1 <= nx:
            raise ValueError(f"slab [{k0}, {k1}) outside the volume's {nx} planes")
        n_views, shift, ev = self._snapshot()
        with torch.cuda.device(self.device), torch.cuda.stream(self.stream):
            slab = torch.empty((k1 - k0, ny, nz), dtype=torch.float32, device=self.device)
            if n_views == 0 or k1 == k0:
                slab.zero_()
            else:
                g = np.zeros(1, dtype=N.GRID_DTYPE)
                g[0] = volume_grid_record(origin, h, dims, k0, k1)
                g["out_offset"] = 0
                g["cor_shift"] = shift
                self._run_grids(g, slab.view(-1), n_views, ev)
        _handoff(self.stream, slab)
        return slab, origin, h

    def reconstruct_volume(self, voxel=None, maxdim=None, chunk=262144, progress=None):
        """Full 3D reconstruction of the volume box on a regular grid.
        Returns (volume [nx, ny, nz] float32, origin (mm), voxel size (mm))."""
        vol, origin, h = self.reconstruct_volume_tensor(voxel, maxdim, None, progress)
        return vol.cpu().numpy(), origin, h

    def preview_volume(self, maxdim=64, chunk=65536):
        return self.reconstruct_volume(maxdim=maxdim, chunk=chunk)

    def device_status(self):
        """Raise TimeoutError if a bounded device-side wait ever gave up (reads one
        int32 after synchronising the reconstruction stream)."""
        self.stream.synchronize()
        code = int(self._status.item())
        if code != 0:
            N.check(code, "device-side status")

    def warmup(self):
        """Load the library and run one tiny back-projection (no JIT involved)."""
        if self.n == 0:
            return
        self.reconstruct_points(np.zeros((4, 3)))

    # ----------------------------------------------------------- rotation centre
    def set_cor_shift(self, px):
        """Take the rotation axis to project `px` detector columns right of nominal."""
        with self._lock:
            self.cor_shift = float(px)
            self.version += 1

    def cor_scores(self, shifts, n=192, z=0.0, bins=128):
        """-entropy of the axial slice at z for every trial shift: one batched
        back-projection of all trial slices, then one scoring launch (mr_slice_entropy)."""
        reqs = [dict(origin=(0.0, 0.0, z), normal=(0.0, 0.0, 1.0), n=n, cor_shift=float(s))
                for s in shifts]
        if not reqs:
            return np.zeros(0)
        out, _ = self._planes(reqs)
        with torch.cuda.device(self.device):
            st = torch.cuda.current_stream(self.device)
            scores = torch.empty(len(reqs), dtype=torch.float64, device=self.device)
            N.check(N.load().mr_slice_entropy(ctypes_void(out.data_ptr()), len(reqs), n * n, n * n, bins,
                                              ctypes_void(scores.data_ptr()), ctypes_void(st.cuda_stream)),
                    "mr_slice_entropy")
            return scores.cpu().numpy()

    def bp_operator(self, requests):
        """A differentiable back-projection (autograd.BackprojectOp) of the given slice
        requests over the current snapshot of views; use with autograd.backproject."""
        from .autograd import BackprojectOp
        n_views, _, ev = self._snapshot()
        if ev is not None:
            torch.cuda.current_stream(self.device).wait_event(ev)
        grids = np.zeros(len(requests), dtype=N.GRID_DTYPE)
        off = 0
        for r, req in enumerate(requests):
            n = int(req.get("n", 256))
            grids[r] = plane_grid(self.box, req["origin"], req["normal"], n, req.get("size"),
                                  req.get("zoom", 1.0), req.get("center"), 0.0)
            grids[r]["out_offset"] = off
            off += n * n
        return BackprojectOp(self._views_dev, self._kind_code, self.geom.rows, self.geom.cols, grids, off,
                             n_views)

    def calibrate(self, shift0=None, tilt0=0.0, z=0.0, n=192, fit_tilt=True, iters=60, tol=1e-3,
                  heights=(-0.6, 0.6), verbose=False):
        """Gradient-based rotation-centre / detector-tilt calibration.

        The score of a set of slices is a differentiable histogram score (Gaussian-kernel
        soft histogram of each slice, the smooth counterpart of the estimate_cor criterion
        sum p log p, recon.py:508-512), maximised by gradient ascent with backtracking; the
        gradients come from the hand-written backward of the back-projector.
          1. the COR shift [px] on the axial slice at z - the plane the grid search of
             estimate_cor scores (recon.py:498-519), which projects onto the central
             detector rows, where an in-plane detector tilt moves nothing - and the central
             x-z slice, whose score moves the ascent off a wrong start (a COR error smears
             every slice);
          2. with fit_tilt, the tilt [deg] with the shift held, on axial slices at
             `heights` x the box half-height: a tilt shows as a COR shift that grows with
             the distance from the central row, so the slices far from it see it most
             (slices near the centre add noise-driven jitter and no tilt signal);
          3. with fit_tilt, the shift again at that tilt; steps 2 and 3 alternate until
             neither moves by more than `tol` (the best tilt of the outer slices depends on
             the shift they are seen with).
        Sets the shift (the tilt is returned, not stored). Returns (shift, tilt_deg,
        history), history a list of (shift, tilt_deg, score) after every step."""
        from .autograd import backproject, soft_neg_entropy
        ring = self._ring
        dev = self.device
        deg = np.pi / 180.0
        zb = float(self.box[2])

        def objective(planes):
            reqs = [dict(origin=o, normal=nrm, n=n) for o, nrm in planes]
            op = self.bp_operator(reqs)
            with torch.no_grad():      # histogram ranges fixed from the nominal geometry
                f0 = backproject(ring, torch.tensor(0.0, dtype=torch.float64),
                                 torch.tensor(0.0, dtype=torch.float64), op)
            ranges = []
            for k in range(len(planes)):
                part = f0[k * n * n:(k + 1) * n * n]
                nz = part[part != 0]
                ranges.append((float(nz.min()), float(nz.max())) if nz.numel() else (0.0, 1.0))

            def score(xv, active):
                xs = xv.clone().requires_grad_(True)
                f = backproject(ring, xs[0], xs[1] * deg, op)
                J = 0.0
                for k, (lo, hi) in enumerate(ranges):
                    J = J + soft_neg_entropy(f[k * n * n:(k + 1) * n * n].double(), lo, hi)
                J.backward()
                g = xs.grad.clone()
                g[1 - active] = 0.0
                return float(J.detach()), g
            return score

        def ascend(score, x, active, hist):
            J, g = score(x, active)
            step = 0.5
            for _ in range(iters):
                gmax = float(g.abs().max())
                if gmax == 0.0:
                    break
                d = g / gmax                                   # unit max-norm ascent direction
                accepted = False
                while step > tol / 4:
                    xn = x + step * d
                    Jn, gn = score(xn, active)
                    if Jn > J:
                        x, J, g = xn, Jn, gn
                        step *= 1.5
                        accepted = True
                        break
                    step *= 0.5
                hist.append((float(x[0]), float(x[1]), J))
                if not accepted or step < tol:
                    break
            return x

        x = torch.tensor([self.cor_shift if shift0 is None else float(shift0), float(tilt0)],
                         dtype=torch.float64, device=dev)
        hist = [(float(x[0]), float(x[1]), float("nan"))]
        axial = (0.0, 0.0, 1.0)
        centre = objective([((0.0, 0.0, z), axial), ((0.0, 0.0, 0.0), (0.0, 1.0, 0.0))])
        x = ascend(centre, x, 0, hist)
        if fit_tilt:
            outer = objective([((0.0, 0.0, h * zb), axial) for h in heights])
            for _ in range(6):
                prev = x.clone()
                x = ascend(outer, x, 1, hist)
                x = ascend(centre, x, 0, hist)
                if float((x - prev).abs().max()) < 10 * tol:
                    break
        self.set_cor_shift(float(x[0]))
        if verbose:
            print(f"[minirecast] calibrated COR shift {float(x[0]):+.3f} px, tilt {float(x[1]):+.4f} deg "
                  f"({len(hist) - 1} steps)")
        return float(x[0]), float(x[1]), hist

    def estimate_cor(self, shifts=None, n=192, z=0.0, verbose=True):
        """Pick the COR shift whose central axial slice has the lowest histogram entropy
        (recon.py:498-519); all trial slices go in one batched launch."""
        if shifts is None:
            shifts = np.arange(-3.0, 3.01, 0.25)
        shifts = np.asarray(shifts, dtype=float)
        scores = self.cor_scores(shifts, n, z)
        best = float(shifts[int(np.argmax(scores))])
        self.set_cor_shift(best)
        if verbose:
            print("[minirecast] COR search: " + " ".join(
                f"{s:+.2f}:{v:.3g}" for s, v in zip(shifts, scores)))
            print(f"[minirecast] best COR shift {best:+.2f} px")
        return best, scores

    def scan_replay(self, raw, requests):
        """Capture the reconstruction of a whole scan held in a device buffer as one CUDA
        graph -> ScanReplay. See ScanReplay."""
        return ScanReplay(self, raw, requests)


class ScanReplay:
    """A resident scan reconstructed by a captured CUDA graph.

    The graph holds the two launches that reconstruct a scan from the device buffer `raw`
    (uint16 counts [k, R0, C0]): the fused ingest of all k views into ring slots 0 .. k-1
    and the batched back-projection of `requests` (reconstruct_planes_tensor's dicts)
    into one device buffer. replay() runs them again with no host work between them, so
    an acquisition that writes each new scan into the same device buffer under a fixed
    protocol (the same orbit, flat / dark fields and slices) is reconstructed at the
    device's pace whatever the host's; `images` are views of the output buffer, and
    replay() returns them. After a replay the reconstructor holds views 0 .. k-1 in
    order, as after reset() and add_raw_projections(arange(k), raw), and serves further
    requests from them. Everything the launches read is bound at capture: the buffer,
    the flat / dark fields (set_flat_dark() afterwards invalidates the replay), the COR
    shift and the requests.
    """

    def __init__(self, rec, raw, requests):
        if not (isinstance(raw, torch.Tensor) and raw.is_cuda and raw.device == rec.device):
            raise ValueError("scan_replay needs the raw counts in a CUDA tensor on the reconstructor's device")
        if raw.element_size() != 2 or raw.ndim != 3 or not raw.is_contiguous():
            raise ValueError("raw counts must be a contiguous 16-bit [k, rows, cols] tensor")
        if getattr(rec, "_gain", None) is None:
            raise RuntimeError("call set_flat_dark() before scan_replay()")
        if rec._parker is not None or rec._proj is not None or rec.gaussian or rec.tilt:
            raise ValueError("scan_replay covers the fused ingest only (no Parker weights, kept "
                             "projections or pre-processing)")
        k = int(raw.shape[0])
        if not 0 < k <= rec.n_total:
            raise ValueError(f"{k} views for a ring of {rec.n_total}")
        b, R, C = rec._raw_bin, rec.geom.rows, rec.geom.cols
        if raw.shape[1] < R * b or raw.shape[2] < C * b:
            raise ValueError(f"raw frames {tuple(raw.shape[1:])} are smaller than {R * b} x {C * b}")
        self.rec, self.k = rec, k
        self.raw = raw.view(torch.int16) if raw.dtype == torch.uint16 else raw
        self._dark, self._gain = rec._dark, rec._gain
        self.indices = np.arange(k)
        dev = rec.device
        # records, bound for the whole life of the graph
        fv_host = rec._filter_views(self.indices, self.indices)
        grids = np.zeros(len(requests), dtype=N.GRID_DTYPE)
        sizes, offset = [], 0
        for r, req in enumerate(requests):
            n = int(req.get("n", 256))
            s_ = req.get("cor_shift")
            grids[r] = rec._plane_record(req["origin"], req["normal"], n, req.get("size"), req.get("zoom", 1.0),
                                         req.get("center"), rec.cor_shift if s_ is None else float(s_))
            grids[r]["out_offset"] = offset
            sizes.append(n)
            offset += n * n
        grids["n_views"] = k
        grids["scale"] = np.pi / k
        tiles = N.plan_tiles(grids, rec._band_axis)
        self.stream = torch.cuda.Stream(dev)
        rec.reset()
        timer, rec.kernel_timer = rec.kernel_timer, None         # no timing events in the graph
        try:
            self._capture(rec, fv_host, grids, tiles, offset)
        finally:
            rec.kernel_timer = timer
        self.images = []
        o = 0
        for n in sizes:
            self.images.append(self.out[o:o + n * n].view(n, n))
            o += n * n
        self.replay()

    def _capture(self, rec, fv_host, grids, tiles, offset):
        dev = rec.device
        with rec._ingest_lock:
            with torch.cuda.device(dev), torch.cuda.stream(self.stream):
                self.fv = torch.from_numpy(fv_host.view(np.uint8).copy()).to(dev)
                recs = np.concatenate([grids.view(np.uint8), tiles.view(np.uint8)])
                self.recs = torch.from_numpy(recs).to(dev)
                self.out = torch.zeros(max(offset, 1), dtype=torch.float32, device=dev)
            self.n_tiles = len(tiles)
            self._g_off = 0
            self._t_off = grids.nbytes
            with torch.cuda.device(dev), torch.cuda.stream(rec.ingest_stream):
                rec._upload_view_records(self.indices, self.indices)
            torch.cuda.synchronize(dev)
            self._launch()                      # once eagerly: module loading, kernel attributes
            torch.cuda.synchronize(dev)
            self.graph = torch.cuda.CUDAGraph()
            with torch.cuda.device(dev):
                with torch.cuda.graph(self.graph, stream=self.stream, capture_error_mode="thread_local"):
                    self._launch()

    def _launch(self):
        rec, st = self.rec, torch.cuda.current_stream(self.rec.device)
        rec._ingest_launch(self.raw, 0, self.k, self.fv, stream=st)
        if self.n_tiles == 0:
            return
        lib, v = N.load(), ctypes_void
        base = self.recs.data_ptr()
        fn = lib.mr_backproject_staged if rec.bp_kernel == "staged" else lib.mr_backproject
        name = "mr_backproject_staged" if rec.bp_kernel == "staged" else "mr_backproject"
        args = [rec._ring_c, v(rec._views_dev.data_ptr()), v(base + self._g_off), v(base + self._t_off),
                self.n_tiles, v(self.out.data_ptr())]
        if rec.bp_kernel == "staged":
            args.append(v(rec._status.data_ptr()))
        N.check(fn(*args, v(st.cuda_stream)), name)

    def replay(self):
        """Filter the buffer's k views into the ring and back-project the requests, on the
        device; returns `images` (f32 [n, n] device tensors, ready on the caller's stream)."""
        rec = self.rec
        if rec._dark is not self._dark or rec._gain is not self._gain:
            raise RuntimeError("set_flat_dark() was called after the capture: make a new scan_replay")
        with rec._ingest_lock, rec._lock:
            with torch.cuda.device(rec.device):
                # the ring's previous readers and writers first; the view records of the
                # slots again if another scan order replaced them meanwhile
                with torch.cuda.stream(rec.ingest_stream):
                    rec._upload_view_records(self.indices, self.indices)
                for other in (rec.stream, rec.ingest_stream):
                    ev = torch.cuda.Event()
                    ev.record(other)
                    self.stream.wait_event(ev)
                with torch.cuda.stream(self.stream):        # a graph runs on the current stream
                    self.graph.replay()
                done = torch.cuda.Event()
                done.record(self.stream)
                rec.stream.wait_event(done)
                rec.ingest_stream.wait_event(done)
            rec._received[:] = False
            rec._received[self.indices] = True
            rec._order[:self.k] = self.indices
            rec._chunk_marks = []
            rec._ingest_event = done
            rec.n = self.k
            rec.version += 1
        _handoff(self.stream, self.out)
        return self.images
