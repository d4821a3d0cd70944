"""Projection pre-processing applied on arrival (minirecast preprocess.py), on the GPU.

Blocks are [rows, k, cols] float32. `gaussian_blur` and `rotate_projections` accept
NumPy (returning NumPy) or CUDA tensors (returning CUDA tensors).
"""
import ctypes

import numpy as np
import torch

from . import _native as N


def _void(x):
    return ctypes.c_void_p(int(x))


def gaussian_taps(n, pad, sigma):
    """Even kernel g of the circular convolution that preprocess.py:21-26 applies over
    a padded axis of length n + 2 pad: g = irfft(exp(-2 (pi f sigma)^2)), FP64. The
    spectrum is cut at Nyquist, so for small sigma g has slowly decaying aliasing tails:
    every tap above 1e-12 of g[0] is kept, up to the full circular length."""
    Np = n + 2 * pad
    f = np.fft.rfftfreq(Np)
    g = np.fft.irfft(np.exp(-2.0 * (np.pi * f * sigma) ** 2), n=Np)
    half = g[:Np // 2 + 1]
    big = np.nonzero(np.abs(half) > 1e-12 * abs(half[0]))[0]
    K = int(big.max()) if big.size else 0
    taps = g[:K + 1].copy()
    if 2 * K == Np:
        taps[K] *= 0.5          # m = +K and m = -K are the same circular tap: count it once
    return taps


def _as_device(block):
    if isinstance(block, torch.Tensor):
        if not block.is_cuda:
            raise ValueError("tensor inputs must live on a CUDA device")
        return block.to(torch.float32).contiguous(), True
    if not torch.cuda.is_available():
        raise RuntimeError("a CUDA device is required: this library has no CPU path")
    t = torch.from_numpy(np.ascontiguousarray(block, dtype=np.float32)).cuda()
    return t, False


def _gaussian_dev(x, sigma):
    R, k, C = x.shape
    pad = int(np.ceil(3 * sigma))
    lib = N.load()
    st = torch.cuda.current_stream(x.device)
    cur = x
    for axis, n in ((0, R), (2, C)):
        taps = torch.from_numpy(gaussian_taps(n, pad, sigma).astype(np.float32)).to(x.device)
        out = torch.empty_like(cur)
        N.check(lib.mr_gaussian_axis_f32(_void(cur.data_ptr()), _void(out.data_ptr()), R, k, C, axis,
                                         pad, _void(taps.data_ptr()), taps.numel(),
                                         _void(st.cuda_stream)), "mr_gaussian_axis_f32")
        taps.record_stream(st)
        cur = out
    return cur


def _rotate_dev(x, degrees):
    R, k, C = x.shape
    out = torch.empty_like(x)
    st = torch.cuda.current_stream(x.device)
    N.check(N.load().mr_rotate_f32(_void(x.data_ptr()), _void(out.data_ptr()), R, k, C,
                                   float(degrees), _void(st.cuda_stream)), "mr_rotate_f32")
    return out


def gaussian_blur(block, sigma):
    """Separable Gaussian low-pass (sigma in detector pixels) on each projection."""
    if sigma <= 0:
        return block
    x, is_t = _as_device(block)
    y = _gaussian_dev(x, float(sigma))
    return y if is_t else y.cpu().numpy()


def rotate_projections(block, degrees):
    """Rotate every projection by `degrees` about the detector centre (bilinear)."""
    if abs(degrees) < 1e-9:
        return block
    x, is_t = _as_device(block)
    y = _rotate_dev(x, degrees)
    return y if is_t else y.cpu().numpy()


def apply(block, gaussian=0.0, tilt=0.0):
    if tilt:
        block = rotate_projections(block, -tilt)
    if gaussian:
        block = gaussian_blur(block, gaussian)
    return block


def apply_device(x, gaussian=0.0, tilt=0.0):
    """Device [rows, k, cols] f32 -> (pre-processed block, view stride, row stride)."""
    if tilt and abs(tilt) >= 1e-9:
        x = _rotate_dev(x, -tilt)
    if gaussian and gaussian > 0:
        x = _gaussian_dev(x, float(gaussian))
    R, k, C = x.shape
    return x, C, k * C
