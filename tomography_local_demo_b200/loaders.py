"""Scan loaders with the correction on the device: minirecast flexray.py (FleX-ray TIFF
folders, cone beam) and hdf5.py (Data Exchange HDF5, parallel beam).

Same call surface and results as the reference loaders (projections [rows, angles, cols]
as -log(I/I0) float32, and the geometry), built the device way:
  * raw uint16 frames are read straight into pinned host buffers (a TIFF reader of
    baseline uncompressed 16-bit strips, PIL for anything else; h5py datasets for HDF5),
    in chunks of views whose upload and correction overlap the reading of the next chunk;
  * the per-projection correction (bin mean, row flip, (P-D)*gain or (P-D)/(F-D), clip,
    -log) and the detector crop run in one CUDA kernel (mr_correct_u16) writing the
    stack in the reference's layout, which stays on the device with as_tensor=True
    (SliceReconstructor consumes it in place);
  * the FleX-ray shadow crop (99th percentiles of 24 sampled projections) and the object
    box (mean detector profiles of all projections) are reduced on the device.
Flat and dark frames (a few per scan) are averaged on the host exactly as the reference
does, so the gain is the same float32 array.
"""
import ctypes
import glob
import os
import re
import struct
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import torch

from . import _native as N
from .geometry import ConeVecGeometry, ParallelGeometry
from .model import linear_neighbours, lerp_like_numpy
from .recon import ctypes_void

# Scanner correction profiles of flexDATA (motor offsets measured by CWI), the same table
# as flexray.py:22-29: the geometry of a scan depends on these numbers.
PROFILES = {
    "none": {},
    "cwi-flexray-2019-04-24": {"det_tan": 24.0, "src_ort": -7.0, "axs_tan": -0.5},
    "cwi-flexray-2020-03-26": {"det_tan": 24.300, "src_ort": -6.086, "axs_tan": -0.524},
    "cwi-flexray-2022-10-28": {"det_tan": 24.0485, "src_ort": -5.7730, "axs_tan": -0.5010},
    "cwi-flexray-2024-07-25": {"det_tan": 24.0042, "src_ort": -6.2879, "axs_tan": -0.5143},
}

_NUMBER = re.compile(r"\s*([-+]?\d*\.?\d+(?:[eE][-+]?\d+)?)")


# ------------------------------------------------------------------ scan settings
def parse_scan_settings(path):
    """Geometry parameters (mm) from 'scan settings.txt' (flexray.py:35-78): "key: value"
    lines, keys case-insensitive, numbers taken from the start of the value; ROI given in
    unbinned pixels of the 1944 x 1536 detector (centre (971, 767), pitch 74.8 um)."""
    fname = os.path.join(path, "scan settings.txt")
    num, text = {}, {}
    with open(fname, "r", errors="replace") as f:
        for line in f:
            key, sep, val = line.partition(":")
            if not sep:
                continue
            key = key.strip().lower()
            text[key] = val.strip()
            m = _NUMBER.match(val)
            num[key] = float(m.group(1)) if m else val.strip()

    def need(k):
        if k not in num:
            raise KeyError(f"'{k}' missing in {fname}")
        return num[k]

    sod, sdd = need("sod"), need("sdd")
    p = dict(src2obj=sod, det2obj=sdd - sod, img_pixel=need("voxel size") / 1000.0,
             src_ort=num.get("ver_tube", 0.0), src_tan=num.get("tra_tube", 0.0),
             det_ort=num.get("ver_det", 0.0), det_tan=num.get("tra_det", 0.0),
             axs_tan=num.get("tra_obj", 0.0), theta_min=num.get("start angle", 0.0),
             theta_max=num.get("last angle", 360.0),
             roi=[int(float(x)) for x in text.get("roi (ltrb)", "0,0,1943,1535").split(",")],
             name=num.get("sample name", ""))
    p["det_pixel"] = p["img_pixel"] * sdd / sod
    roi = p["roi"]
    p["det_tan"] += ((roi[0] + roi[2]) // 2 - 971) * 0.0748
    p["det_ort"] += ((roi[1] + roi[3]) // 2 - 767) * 0.0748
    return p


def cone_vectors(p, thetas_deg, pixel):
    """ASTRA cone_vec rows of a circular FleX-ray orbit about +z (flexray.py:81-96): source
    at -y rotated by theta, detector centre across the axis, volume centred vertically
    between source and detector height."""
    z0 = (p["det_ort"] * p["src2obj"] + p["src_ort"] * p["det2obj"]) / (p["src2obj"] + p["det2obj"])
    th = np.deg2rad(np.asarray(thetas_deg, dtype=float))
    c, s = np.cos(th), np.sin(th)

    def rot(x, y):
        return np.stack([c * x - s * y, s * x + c * y], axis=1)

    V = np.zeros((len(th), 12))
    V[:, 0:2] = rot(p["src_tan"] - p["axs_tan"], -p["src2obj"])
    V[:, 2] = p["src_ort"] - z0
    V[:, 3:5] = rot(p["det_tan"] - p["axs_tan"], p["det2obj"])
    V[:, 5] = p["det_ort"] - z0
    V[:, 6:8] = rot(pixel, 0.0)
    V[:, 11] = pixel
    return V


# ------------------------------------------------------------------ TIFF frames
_TIFF_TYPES = {3: ("H", 2), 4: ("I", 4)}


def _tiff_strips(f):
    """(byte order, width, height, [(offset, bytes)]) of a baseline uncompressed 16-bit
    single-channel unsigned TIFF (the first image), or None for any other kind."""
    head = f.read(8)
    if len(head) < 8 or head[:2] not in (b"II", b"MM"):
        return None
    e = "<" if head[:2] == b"II" else ">"
    if struct.unpack(e + "H", head[2:4])[0] != 42:
        return None
    f.seek(struct.unpack(e + "I", head[4:8])[0])
    n = struct.unpack(e + "H", f.read(2))[0]
    raw = f.read(12 * n)
    tags = {}
    for i in range(n):
        tag, typ, cnt, val = struct.unpack(e + "HHI4s", raw[12 * i:12 * i + 12])
        if typ not in _TIFF_TYPES or cnt == 0:
            continue
        code, size = _TIFF_TYPES[typ]
        if cnt * size <= 4:
            tags[tag] = struct.unpack(e + code * cnt, val[:cnt * size])
        else:
            pos = f.tell()
            f.seek(struct.unpack(e + "I", val)[0])
            tags[tag] = struct.unpack(e + code * cnt, f.read(cnt * size))
            f.seek(pos)
    one = lambda t, d: tags.get(t, (d,))[0]        # noqa: E731
    w, h = one(256, 0), one(257, 0)
    if (one(258, 1) != 16 or one(259, 1) != 1 or one(277, 1) != 1 or one(339, 1) != 1
            or one(262, 1) != 1 or w <= 0 or h <= 0):
        return None
    offs, cnts = tags.get(273), tags.get(279)
    if not offs or not cnts or len(offs) != len(cnts) or sum(cnts) != 2 * w * h:
        return None
    return e, w, h, list(zip(offs, cnts))


def tiff_shape(fname):
    """(height, width) of a 16-bit frame (PIL when the fast reader does not apply)."""
    with open(fname, "rb") as f:
        lay = _tiff_strips(f)
    if lay is not None:
        return lay[2], lay[1]
    return _imread_pil(fname).shape


def _imread_pil(fname):
    from PIL import Image
    return np.array(Image.open(fname))


def read_tiff_u16(fname, out=None):
    """uint16 frame of a TIFF file, read straight into `out` (a C-contiguous uint16 array,
    e.g. a view of a pinned buffer) when given. Baseline uncompressed strips are read with
    readinto (no intermediate copy); other TIFFs go through PIL, like the reference's
    fallback (flexray.py:102-108)."""
    with open(fname, "rb", buffering=0) as f:
        lay = _tiff_strips(f)
        if lay is not None:
            e, w, h, strips = lay
            if out is None:
                out = np.empty((h, w), np.uint16)
            elif out.shape != (h, w) or out.dtype != np.uint16 or not out.flags.c_contiguous:
                raise ValueError(f"{fname}: frame is {h}x{w}, buffer {out.shape} {out.dtype}")
            buf = memoryview(out.reshape(-1).view(np.uint8))
            pos = 0
            for off, cnt in strips:
                f.seek(off)
                if f.readinto(buf[pos:pos + cnt]) != cnt:
                    raise ValueError(f"{fname}: truncated image data")
                pos += cnt
            if e == ">":
                out.byteswap(inplace=True)
            return out
    im = _imread_pil(fname)
    if out is None:
        return im
    if im.shape != out.shape:
        raise ValueError(f"{fname}: frame is {im.shape}, buffer {out.shape}")
    out[...] = im
    return out


def _read_binned(fname, sample):
    """Binned float32 frame, rows bottom-up (flexray.py:111-116): float32 mean of
    sample x sample blocks, then flipped upside down."""
    im = read_tiff_u16(fname).astype(np.float32)
    if sample > 1:
        h, w = (im.shape[0] // sample) * sample, (im.shape[1] // sample) * sample
        im = im[:h, :w].reshape(h // sample, sample, w // sample, sample).mean(axis=(1, 3))
    return np.flipud(im)


def _files(path, prefix):
    return sorted(f for f in glob.glob(os.path.join(path, prefix + "*"))
                  if f.lower().endswith((".tif", ".tiff")))


# ------------------------------------------------------------------ device helpers
def _device(device):
    return torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())


def _correct(raw_dev, k, bin_, flip, rows_full, row0, col0, rows, cols, dark_dev, scale_dev, mode, out, so_row,
             so_view, stream):
    """mr_correct_u16 of k device frames raw_dev [k, H0, W0] (uint16 bits) into `out`."""
    v = ctypes_void
    st = N.load().mr_correct_u16(v(raw_dev.data_ptr()), raw_dev.shape[1] * raw_dev.shape[2], raw_dev.shape[2], k,
                                 bin_, int(flip), rows_full, row0, col0, rows, cols, v(dark_dev.data_ptr()),
                                 v(scale_dev.data_ptr()), dark_dev.shape[1], mode, v(out.data_ptr()), so_row,
                                 so_view, v(stream.cuda_stream))
    N.check(st, "mr_correct_u16")


class _FrameStream:
    """Reads frames (a callable filling a uint16 [k, H0, W0] numpy view) into two pinned
    buffers in turn; each chunk is uploaded and corrected on `stream` while the host
    reads the next one."""

    def __init__(self, h0, w0, chunk, device, stream):
        self.chunk = chunk
        self.stream = stream
        self.pinned = [torch.empty((chunk, h0, w0), dtype=torch.int16).pin_memory() for _ in range(2)]
        self.staged = [torch.empty((chunk, h0, w0), dtype=torch.int16, device=device) for _ in range(2)]
        self.done = [None, None]

    def run(self, n, fill, consume):
        """fill(i0, i1, host_u16) reads views [i0, i1); consume(i0, i1, device_frames)
        queues their correction on the stream."""
        for j, i0 in enumerate(range(0, n, self.chunk)):
            i1 = min(n, i0 + self.chunk)
            b = j % 2
            if self.done[b] is not None:
                self.done[b].synchronize()          # the buffer's previous chunk has left
            host = self.pinned[b][:i1 - i0]
            fill(i0, i1, host.numpy().view(np.uint16))
            with torch.cuda.stream(self.stream):
                dev = self.staged[b][:i1 - i0]
                dev.copy_(host, non_blocking=True)
                consume(i0, i1, dev)
                ev = torch.cuda.Event()
                ev.record(self.stream)
            self.done[b] = ev
        self.stream.synchronize()


def _shadow_range(profile, frac=0.1, pad=16):
    """[start, stop) of the detector range whose profile exceeds frac * max, padded
    (flexray.py:147-151)."""
    idx = np.nonzero(profile > frac * profile.max())[0]
    if idx.size == 0:
        return 0, len(profile)
    return max(0, idx[0] - pad), min(len(profile), idx[-1] + 1 + pad)


def _percentile_along(t, q, dim):
    """numpy.percentile(x, q, axis=dim) of a float32 device tensor: the two neighbouring
    order statistics of every lane (a device sort) blended on the host as numpy does."""
    n = t.shape[dim]
    prev, nxt, gamma = linear_neighbours(n, [q])
    s = torch.sort(t, dim=dim).values
    a = s.select(dim, int(prev[0])).cpu().numpy()
    b = s.select(dim, int(nxt[0])).cpu().numpy()
    return lerp_like_numpy(a, b, gamma[0])


def object_box(proj, V, full_box, margin=1.15):
    """Tight half-size box (mm) around the object from its shadow on the detector
    (flexray.py:124-144), with the mean detector profiles of a device stack
    [rows, angles, cols] reduced on the device (FP64 sums)."""
    if isinstance(proj, torch.Tensor):
        cnt_c = proj.shape[0] * proj.shape[1]
        cnt_r = proj.shape[1] * proj.shape[2]
        col_prof = (torch.sum(proj, dim=(0, 1), dtype=torch.float64) / cnt_c).cpu().numpy()
        row_prof = (torch.sum(proj, dim=(1, 2), dtype=torch.float64) / cnt_r).cpu().numpy()
        cols_total = proj.shape[2]
        rows_total = proj.shape[0]
    else:
        col_prof = proj.mean(axis=(0, 1))
        row_prof = proj.mean(axis=(1, 2))
        cols_total, rows_total = proj.shape[2], proj.shape[0]
    cols = np.nonzero(col_prof > 0.03 * col_prof.max())[0]
    rows = np.nonzero(row_prof > 0.03 * row_prof.max())[0]
    if cols.size == 0 or rows.size == 0:
        return full_box
    s, d, u, v = V[0, 0:3], V[0, 3:6], V[0, 6:9], V[0, 9:12]
    n = np.cross(u, v)
    n /= np.linalg.norm(n)
    mag = abs((d - s) @ n) / abs(-s @ n)
    t = ((d - s) @ n) / ((-s) @ n)
    hit = s + t * (-s) - d
    c0 = hit @ u / (u @ u) + (cols_total - 1) / 2
    r0 = hit @ v / (v @ v) + (rows_total - 1) / 2
    pu, pv = np.linalg.norm(u), np.linalg.norm(v)
    rxy = max(abs(cols[0] - c0), abs(cols[-1] - c0)) * pu / mag
    rz = max(abs(rows[0] - r0), abs(rows[-1] - r0)) * pv / mag
    box = np.array([rxy, rxy, rz]) * margin + 1.0
    return np.minimum(box, full_box)


# ------------------------------------------------------------------ FleX-ray
def load_flexray(path, sample=4, skip=2, profile="cwi-flexray-2019-04-24", threads=8, auto_box=True, crop=True,
                 verbose=True, device=None, as_tensor=False, chunk=32):
    """Return (projections [rows, angles, cols] as -log(I/I0), ConeVecGeometry), like
    flexray.py:154-225. as_tensor=True returns the stack as a CUDA tensor (no copy back);
    chunk = views per upload / correction launch."""
    path = os.path.expanduser(path)
    p = parse_scan_settings(path)
    for k, val in PROFILES[profile].items():
        p[k] += val

    scans = _files(path, "scan_")
    if not scans:
        raise FileNotFoundError(f"no scan_*.tif files in {path}")
    n_total = len(scans)
    scans = scans[::skip]
    dark = np.mean([_read_binned(f, sample) for f in _files(path, "di")], axis=0)
    flat = np.mean([_read_binned(f, sample) for f in _files(path, "io")], axis=0)
    gain = 1.0 / np.maximum(flat - dark, 1.0)
    R_full, C_full = dark.shape
    h0, w0 = tiff_shape(scans[0])
    if (h0 // sample, w0 // sample) != (R_full, C_full):
        raise ValueError(f"scan frames {h0}x{w0} do not match the flat/dark frames")

    dev = _device(device)
    with torch.cuda.device(dev):
        stream = torch.cuda.Stream(dev)
        dark_d = torch.from_numpy(np.ascontiguousarray(dark, dtype=np.float32)).to(dev)
        gain_d = torch.from_numpy(np.ascontiguousarray(gain, dtype=np.float32)).to(dev)
        pool = ThreadPoolExecutor(max(1, int(threads)))

        def fill_from(files):
            def fill(i0, i1, host):
                list(pool.map(lambda j: read_tiff_u16(files[i0 + j], host[j]), range(i1 - i0)))
            return fill

        frames = _FrameStream(h0, w0, max(1, min(int(chunk), len(scans))), dev, stream)
        try:
            r0, r1, c0, c1 = 0, R_full, 0, C_full
            if crop:
                sample_idx = np.linspace(0, len(scans) - 1, min(24, len(scans))).astype(int)
                picked = [scans[i] for i in sample_idx]
                some = torch.empty((len(picked), R_full, C_full), dtype=torch.float32, device=dev)

                def corr_some(i0, i1, d):
                    _correct(d, i1 - i0, sample, True, R_full, 0, 0, R_full, C_full, dark_d, gain_d,
                             N.MR_CORRECT_FLEXRAY, some[i0:i1], C_full, R_full * C_full, stream)

                frames.run(len(picked), fill_from(picked), corr_some)
                # strongest attenuation per detector row / column over the sampled angles
                # (99th percentile across the other axis), flexray.py:190-197
                r0, r1 = _shadow_range(_percentile_along(some, 99, 2).max(axis=0))
                c0, c1 = _shadow_range(_percentile_along(some, 99, 1).max(axis=0))
                del some
            rows, cols, A = r1 - r0, c1 - c0, len(scans)
            proj = torch.empty((rows, A, cols), dtype=torch.float32, device=dev)

            def corr_all(i0, i1, d):
                _correct(d, i1 - i0, sample, True, R_full, r0, c0, rows, cols, dark_d, gain_d,
                         N.MR_CORRECT_FLEXRAY, proj[:, i0:i1, :], A * cols, cols, stream)

            frames.run(A, fill_from(scans), corr_all)
        finally:
            pool.shutdown()

    step = (p["theta_max"] - p["theta_min"]) / n_total
    thetas = p["theta_min"] + np.arange(0, n_total, skip)[:A] * step
    pixel = p["det_pixel"] * sample
    V = cone_vectors(p, thetas, pixel)
    dc = (c0 + c1 - 1) / 2.0 - (C_full - 1) / 2.0          # the crop moves the detector centre
    dr = (r0 + r1 - 1) / 2.0 - (R_full - 1) / 2.0
    V[:, 3:6] += dc * V[:, 6:9] + dr * V[:, 9:12]
    vox = p["img_pixel"] * sample
    box = np.array([C_full * vox / 2, C_full * vox / 2, R_full * vox / 2])
    if auto_box:
        box = object_box(proj, V, box)
    rng = np.deg2rad(p["theta_max"] - p["theta_min"])
    geom = ConeVecGeometry(V, rows, cols, angular_range=rng, box=box)
    if verbose:
        mb = proj.numel() * 4 / 1e6
        print(f"[flexray] {p['name'] or os.path.basename(path)}: {A}/{n_total} "
              f"projections, {R_full}x{C_full} px after {sample}x{sample} binning, "
              f"cropped to {rows}x{cols} ({mb:.0f} MB)")
        print(f"[flexray] SOD={p['src2obj']:.1f} mm  SDD={p['src2obj'] + p['det2obj']:.1f} mm  "
              f"voxel={vox * 1000:.0f} um  profile={profile}")
        print(f"[flexray] view box (half sizes) = {np.round(box, 1)} mm")
    return (proj if as_tensor else proj.cpu().numpy()), geom


# ------------------------------------------------------------------ Data Exchange HDF5
PIXEL_SIZE_KEYS = (
    "measurement/instrument/detection_system/objective/resolution",
    "measurement/instrument/detector/pixel_size",
    "measurement/instrument/detector/pixel_size_x",
)


def _bin_host(a, sample):
    """Mean of sample x sample blocks of the last two axes (hdf5.py:24-31): float64 mean
    for integer input, rounded to float32."""
    if sample <= 1:
        return a.astype(np.float32)
    *lead, h, w = a.shape
    h2, w2 = (h // sample) * sample, (w // sample) * sample
    a = a[..., :h2, :w2].reshape(*lead, h2 // sample, sample, w2 // sample, sample)
    return a.mean(axis=(-1, -3)).astype(np.float32)


def _read_pixel_size(f):
    for key in PIXEL_SIZE_KEYS:
        if key in f:
            v = float(np.ravel(f[key][()])[0])
            if v > 0:
                return v / 1000.0 if v > 0.05 else v
    return None


def _percentile_all_nonneg(t, q):
    """numpy.percentile(x, q) over every element of a non-negative float32 device tensor:
    exact order statistics of the non-zero elements (mr_volume_select), the zeros below."""
    lib = N.load()
    flat = t.reshape(-1)
    n = flat.numel()
    v = ctypes_void
    dev = flat.device
    ws = torch.empty(int(lib.mr_volume_workspace_bytes()), dtype=torch.uint8, device=dev)
    stats = (ctypes.c_uint64 * 3)()
    stream = torch.cuda.current_stream(dev)
    N.check(lib.mr_volume_stats(v(flat.data_ptr()), n, v(ws.data_ptr()), stats, v(stream.cuda_stream)),
            "mr_volume_stats")
    nonzero, keys = int(stats[0]), int(stats[2])
    zeros = n - nonzero
    out = torch.empty(4, dtype=torch.float32, device=dev)
    prev, nxt, gamma = linear_neighbours(n, [q])

    def value(rank):
        if rank < zeros:
            return np.float32(0.0)
        r = (ctypes.c_int64 * 1)(int(rank - zeros))
        N.check(lib.mr_volume_select(v(flat.data_ptr()), n, r, 1, keys & 0xFFFFFFFF, keys >> 32, v(ws.data_ptr()),
                                     v(out.data_ptr()), v(stream.cuda_stream)), "mr_volume_select")
        return out[0].item()

    return float(lerp_like_numpy(value(int(prev[0])), value(int(nxt[0])), gamma[0]))


def load_dxchange(path, sample=2, skip=1, rows=None, pixel_size=None, h5=None, verbose=True, device=None,
                  as_tensor=False, chunk=32):
    """Return (projections [rows, angles, cols] as -log(I/I0), ParallelGeometry), like
    hdf5.py:43-96; uint16 data is binned and corrected on the device (other dtypes on
    the host, as the reference does). as_tensor=True returns a CUDA tensor."""
    if h5 is None:
        try:
            import h5py
        except ImportError as e:
            raise SystemExit("h5py is not installed - run ./setup.sh again") from e
        h5 = h5py
    r0, r1 = None, None
    if rows:
        a, _, b = str(rows).partition(":")
        r0, r1 = int(a) if a else None, int(b) if b else None
    dev = _device(device)
    with h5.File(path, "r") as f:
        data = f["exchange/data"]
        n_all = data.shape[0]
        rsl = slice(r0, r1)
        raw = np.asarray(data[::skip, rsl, :])                                   # [A, H, W]
        flat = (_bin_host(np.asarray(f["exchange/data_white"][:, rsl, :]), sample).mean(0)
                if "exchange/data_white" in f else None)
        dark = (_bin_host(np.asarray(f["exchange/data_dark"][:, rsl, :]), sample).mean(0)
                if "exchange/data_dark" in f else None)
        if "exchange/theta" in f:
            theta = np.asarray(f["exchange/theta"][()], dtype=float)[::skip]
        else:
            theta = np.linspace(0.0, 180.0, n_all, endpoint=False)[::skip]
        px = pixel_size or _read_pixel_size(f) or 1.0
    A = raw.shape[0]
    H, W = raw.shape[1], raw.shape[2]
    R, C = (H // sample, W // sample) if sample > 1 else (H, W)
    with torch.cuda.device(dev):
        stream = torch.cuda.current_stream(dev)
        if raw.dtype == np.uint16:
            if dark is None:
                dark = np.zeros((R, C), np.float32)
            if flat is None:
                # np.full(..., percentile(binned projections, 99.9)): binned on the device
                t = torch.from_numpy(raw.view(np.int16)).to(dev).to(torch.int32) & 0xFFFF
                b = sample if sample > 1 else 1
                t = t[:, :R * b, :C * b].reshape(A, R, b, C, b).to(torch.float64).mean(dim=(2, 4))
                flat = np.full((R, C), _percentile_all_nonneg(t.to(torch.float32), 99.9), np.float32)
                del t
            denom = np.maximum(flat - dark, 1e-6)
            dark_d = torch.from_numpy(np.ascontiguousarray(dark, dtype=np.float32)).to(dev)
            den_d = torch.from_numpy(np.ascontiguousarray(denom, dtype=np.float32)).to(dev)
            proj = torch.empty((R, A, C), dtype=torch.float32, device=dev)
            raw16 = raw.view(np.int16)
            frames = _FrameStream(H, W, max(1, min(int(chunk), A)), dev, stream)

            def fill(i0, i1, host):
                host[...] = raw16[i0:i1].view(np.uint16)

            def corr(i0, i1, d):
                _correct(d, i1 - i0, sample if sample > 1 else 1, False, R, 0, 0, R, C, dark_d, den_d,
                         N.MR_CORRECT_HDF5, proj[:, i0:i1, :], A * C, C, stream)

            frames.run(A, fill, corr)
        else:
            binned = _bin_host(raw, sample)
            if dark is None:
                dark = np.zeros(binned.shape[1:], np.float32)
            if flat is None:
                flat = np.full(binned.shape[1:], float(np.percentile(binned, 99.9)), np.float32)
            trans = (binned - dark) / np.maximum(flat - dark, 1e-6)
            host = -np.log(np.clip(trans, 1e-3, None)).astype(np.float32)
            proj = torch.from_numpy(np.ascontiguousarray(np.transpose(host, (1, 0, 2)))).to(dev)
    theta = theta[:A]
    span = np.ptp(theta) * len(theta) / max(len(theta) - 1, 1)
    if not (170 < span < 190 or 350 < span < 370):
        print(f"warning: angles cover {span:.0f} deg; FBP assumes 180 or 360")
    pixel = px * sample
    geom = ParallelGeometry(np.deg2rad(theta), proj.shape[0], proj.shape[2], pixel, pixel)
    if verbose:
        unit = "mm" if px != 1.0 else "px (no pixel size in file; use --pixel-size)"
        print(f"[hdf5] {path}: {A}/{n_all} projections, "
              f"{proj.shape[0]}x{proj.shape[2]} after {sample}x{sample} binning, "
              f"pixel {pixel:g} {unit}, angles {theta[0]:.1f}..{theta[-1]:.1f} deg")
    return (proj if as_tensor else proj.cpu().numpy()), geom
