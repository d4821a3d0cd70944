"""TEST INFRASTRUCTURE ONLY. NumPy restatement of minirecast's projection filter path.

Each function follows the cited reference lines; `exact64=True` variants keep every
intermediate in float64 (the FP64 oracle) instead of the reference's float32 casts.
"""
import numpy as np


def ramp_response(n, tau, window="shepp-logan"):
    """recon.py:34-55 - spectrum of the Kak & Slaney discrete ramp kernel."""
    N = int(2 ** np.ceil(np.log2(2 * n)))
    k = np.arange(N)
    idx = np.where(k < N // 2, k, k - N)
    h = np.zeros(N)
    h[0] = 1.0 / (4.0 * tau * tau)
    odd = (idx % 2) == 1
    h[odd] = -1.0 / (np.pi * idx[odd] * tau) ** 2
    H = np.fft.fft(h).real * tau
    f = np.fft.fftfreq(N)
    window_fn = {None: lambda f: 1.0, "ram-lak": lambda f: 1.0, "none": lambda f: 1.0,
                 "shepp-logan": np.sinc,
                 "hann": lambda f: 0.5 * (1.0 + np.cos(2.0 * np.pi * f)),
                 "cosine": lambda f: np.cos(np.pi * f)}
    if window not in window_fn:
        raise ValueError(f"unknown filter window {window!r}")
    return H * window_fn[window](f), N


def filter_rows(data, tau, window="shepp-logan", exact64=False):
    """recon.py:58-64 - rfft(n=N) * H[:N/2+1], irfft, crop, float32 out.
    The FFT runs in the input's precision as in the reference (float32 input ->
    complex64 spectrum on NumPy 2.x); exact64 forces float64 and skips the cast."""
    n = data.shape[-1]
    H, N = ramp_response(n, tau, window)
    x = np.asarray(data, dtype=np.float64) if exact64 else data
    spec = np.fft.rfft(x, n=N, axis=-1)
    spec *= H[: N // 2 + 1]
    y = np.fft.irfft(spec, n=N, axis=-1)[..., :n]
    return y if exact64 else y.astype(np.float32)


def cone_constants(vectors):
    """recon.py:70-82."""
    V = np.asarray(vectors, dtype=np.float64)
    s, d, u, v = (V[:, 3 * i:3 * i + 3] for i in range(4))
    nrm = np.cross(u, v)
    nrm = nrm / np.linalg.norm(nrm, axis=1)[:, None]
    nrm = nrm * np.sign(np.sum((d - s) * nrm, axis=1))[:, None]
    return dict(s=s, d=d, u=u, v=v,
                uu=u / np.sum(u * u, axis=1)[:, None], vv=v / np.sum(v * v, axis=1)[:, None],
                n=nrm, sdd=np.sum((d - s) * nrm, axis=1), sod=np.sum(-s * nrm, axis=1))


def fdk_filter_block(block, K, window="shepp-logan", exact64=False):
    """recon.py:85-104 - per view: FDK cosine weight then ramp filter.
    block [rows, k, cols] -> [k, rows, cols]."""
    R, A, C = block.shape
    cc = np.arange(C) - (C - 1) / 2.0
    rr = np.arange(R) - (R - 1) / 2.0
    out = np.empty((A, R, C), dtype=np.float64 if exact64 else np.float32)
    for k in range(A):
        s, d, u, v, nrm = (K[key][k] for key in ("s", "d", "u", "v", "n"))
        sdd, sod = K["sdd"][k], K["sod"][k]
        off = d - (s + sdd * nrm)
        un, vn = np.linalg.norm(u), np.linalg.norm(v)
        a = off @ u / un + cc * un
        b = off @ v / vn + rr * vn
        w = sdd / np.sqrt(sdd ** 2 + a[None, :] ** 2 + b[:, None] ** 2)
        x = block[:, k, :]
        out[k] = filter_rows(x * w, un * sod / sdd, window, exact64=exact64)
    return out


def parallel_filter_block(block, pixel_u, window="shepp-logan", exact64=False):
    """recon.py:359 - parallel-beam filter of a [rows, k, cols] block -> [k, rows, cols]."""
    return np.transpose(filter_rows(block, pixel_u, window, exact64=exact64), (1, 0, 2))


# ----------------------------------------------------------------- raw correction
def bin_mean(a, sample):
    """hdf5.py:24-31 / flexray.py:111-116 - mean of sample x sample blocks, float32."""
    a = np.asarray(a)
    if sample <= 1:
        return a.astype(np.float32)
    h, w = a.shape[-2] // sample * sample, a.shape[-1] // sample * sample
    a = a[..., :h, :w].astype(np.float32)
    shp = a.shape[:-2] + (h // sample, sample, w // sample, sample)
    return a.reshape(shp).mean(axis=(-1, -3)).astype(np.float32)


def flexray_correct(raw, dark_frames, flat_frames, sample):
    """flexray.py:111-116 + 174-184: binned (and row-flipped) frames, dark/flat means,
    gain = 1/max(F-D, 1), clip at 1e-3, -log. raw [k, R0, C0] uint16 -> [k, R, C] f32."""
    def binned(im):
        return np.flipud(bin_mean(im, sample))
    dark = np.mean([binned(f) for f in dark_frames], axis=0)
    flat = np.mean([binned(f) for f in flat_frames], axis=0)
    gain = 1.0 / np.maximum(flat - dark, 1.0)
    out = []
    for im in raw:
        x = (binned(im) - dark) * gain
        out.append(-np.log(np.clip(x, 1e-3, None)))
    return np.stack(out).astype(np.float32), dark.astype(np.float32), gain.astype(np.float32)


def hdf5_correct(raw, flat_frames, dark_frames, sample):
    """hdf5.py:63-78: trans = (P-D)/max(F-D, 1e-6), clip at 1e-3, -log.
    raw [k, R0, C0] -> [k, R, C] f32."""
    proj = bin_mean(raw, sample)
    flat = bin_mean(np.asarray(flat_frames), sample).mean(0)
    dark = bin_mean(np.asarray(dark_frames), sample).mean(0)
    trans = (proj - dark) / np.maximum(flat - dark, 1e-6)
    return -np.log(np.clip(trans, 1e-3, None)).astype(np.float32), dark, flat


# ----------------------------------------------------------------- preprocess
def gaussian_blur(block, sigma):
    """preprocess.py:8-28 - per axis (rows, then cols): edge pad ceil(3 sigma), FFT
    multiply by exp(-2 (pi f sigma)^2), crop, float32."""
    if sigma <= 0:
        return block
    out = np.array(block, dtype=np.float32)
    pad = int(np.ceil(3 * sigma))
    for axis in (0, 2):
        n = out.shape[axis]
        widths = [(0, 0), (0, 0), (0, 0)]
        widths[axis] = (pad, pad)
        x = np.pad(out, widths, mode="edge")
        Np = x.shape[axis]
        H = np.exp(-2.0 * (np.pi * np.fft.rfftfreq(Np) * sigma) ** 2)
        shape = [1, 1, 1]
        shape[axis] = H.size
        y = np.fft.irfft(np.fft.rfft(x, axis=axis) * H.reshape(shape), n=Np, axis=axis)
        out = np.take(y, np.arange(pad, pad + n), axis=axis).astype(np.float32)
    return out


def rotate_projections(block, degrees):
    """preprocess.py:31-56 - bilinear rotation about the detector centre, zero outside."""
    if abs(degrees) < 1e-9:
        return block
    R, A, C = block.shape
    t = np.deg2rad(degrees)
    rr, cc = np.meshgrid(np.arange(R) - (R - 1) / 2.0, np.arange(C) - (C - 1) / 2.0, indexing="ij")
    rs = np.cos(t) * rr + np.sin(t) * cc + (R - 1) / 2.0
    cs = -np.sin(t) * rr + np.cos(t) * cc + (C - 1) / 2.0
    r0, c0 = np.floor(rs).astype(int), np.floor(cs).astype(int)
    fr, fc = (rs - r0)[..., None], (cs - c0)[..., None]
    out = np.zeros((R, C, A), dtype=np.float32)
    for dr, wr in ((0, 1 - fr), (1, fr)):
        for dc, wc in ((0, 1 - fc), (1, fc)):
            ri, ci = r0 + dr, c0 + dc
            ok = (ri >= 0) & (ri < R) & (ci >= 0) & (ci < C)
            vals = np.zeros((R, C, A), dtype=np.float32)
            vals[ok] = block[ri[ok], :, ci[ok]]
            out += (wr * wc * vals).astype(np.float32)
    return np.ascontiguousarray(np.transpose(out, (0, 2, 1)))


def preprocess_apply(block, gaussian=0.0, tilt=0.0):
    """preprocess.py:59-64 - rotate by -tilt, then Gaussian."""
    if tilt:
        block = rotate_projections(block, -tilt)
    if gaussian:
        block = gaussian_blur(block, gaussian)
    return block
