"""Host side of the tensor-core Toeplitz filter (no GPU): the operand image written by
mr_toeplitz_image decodes, through its SWIZZLE_128B K-major layout, to the split 16-bit
Toeplitz blocks of t_scale * g, g = ifft(H); and the block scheme the kernel evaluates
(x_hi g_hi on every block, hi/lo cross terms on the three diagonals |J - I| <= 1, exact
products, FP32-class sums) reproduces the reference's row filter (recon.py:34-64): to
~1e-5 with FP16 parts, and only to ~5e-4 with BF16 parts on smooth rows, where the ramp
filter's output is ~400 times smaller than its input."""
import numpy as np
import pytest

from oracle import filter as of
from tomography_local_demo_b200 import _native as N
from tomography_local_demo_b200 import build as B
from tomography_local_demo_b200 import recon as R


@pytest.fixture(scope="module")
def lib():
    import os
    if not os.path.exists(B.LIBPATH):
        B.build()
    return N.load()


def bf16(x):
    """Round-to-nearest-even FP32 -> BF16, as float64."""
    f = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    f = (f + 0x7FFF + ((f >> 16) & 1)) >> 16
    return (f.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def f16(x):
    return np.asarray(np.asarray(x, np.float32), np.float16).astype(np.float64)


def decode(img, n_rows, fmt):
    """n_rows x 64 values of a SWIZZLE_128B K-major image of 16-bit elements."""
    u16 = img.view(np.uint16)
    row = np.arange(n_rows)[:, None]
    k = np.arange(64)[None, :]
    off = (row >> 3) * 1024 + (row & 7) * 128 + ((((k >> 3) ^ (row & 7)) & 7) << 4) + (k & 7) * 2
    bits = u16[off // 2]
    if fmt == N.MR_F16:
        return bits.view(np.float16).astype(np.float64)
    return (bits.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def tables(cols, window):
    H, n_fft = R.ramp_response(cols, 1.0, window)
    half = H[: n_fft // 2 + 1]
    full = np.concatenate([half, half[1:n_fft - n_fft // 2][::-1]])
    return np.ascontiguousarray(np.fft.ifft(full).real), n_fft


def build_image(lib, g, n_fft, cols, fmt):
    import ctypes
    img = np.zeros(lib.mr_toeplitz_image_bytes(cols), np.uint8)
    ts = ctypes.c_float()
    assert lib.mr_toeplitz_image(g.ctypes.data, n_fft, cols, fmt, img.ctypes.data, ctypes.byref(ts)) == N.MR_OK
    return img, ts.value


@pytest.mark.parametrize("fmt", [N.MR_F16, N.MR_BF16])
@pytest.mark.parametrize("cols", [64, 100, 486])
def test_image_layout_is_the_split_toeplitz_blocks(lib, cols, fmt):
    g, n_fft = tables(cols, "shepp-logan")
    kb = (cols + 63) // 64
    assert lib.mr_toeplitz_image_bytes(cols) == (2 * kb + 2) * 8192
    img, ts = build_image(lib, g, n_fft, cols, fmt)
    assert 2 ** 13 <= np.abs(g).max() * ts < 2 ** 14 and np.log2(ts) == int(np.log2(ts))
    rnd = f16 if fmt == N.MR_F16 else bf16
    hi = decode(img[: (2 * kb - 1) * 8192], (2 * kb - 1) * 64, fmt)
    lo = decode(img[(2 * kb - 1) * 8192:], 192, fmt)
    r = np.arange(64)[:, None]
    k = np.arange(64)[None, :]
    for d in range(-(kb - 1), kb):
        want = g[(64 * d + r - k) % n_fft] * ts
        np.testing.assert_array_equal(hi[(d + kb - 1) * 64:(d + kb) * 64], rnd(want))
        if abs(d) <= 1:
            np.testing.assert_array_equal(lo[(d + 1) * 64:(d + 2) * 64], rnd(want - rnd(want)))


def test_image_argument_checks(lib):
    import ctypes
    g = np.zeros(1024)
    buf = np.zeros(16, np.uint8)
    ts = ctypes.c_float()
    assert lib.mr_toeplitz_image_bytes(513) == -1
    assert lib.mr_toeplitz_image(g.ctypes.data, 1000, 100, N.MR_F16, buf.ctypes.data, ctypes.byref(ts)) == N.MR_ERR_INVALID
    assert lib.mr_toeplitz_image(g.ctypes.data, 128, 100, N.MR_F16, buf.ctypes.data, ctypes.byref(ts)) == N.MR_ERR_INVALID
    assert lib.mr_toeplitz_image(g.ctypes.data, 1024, 100, N.MR_F32, buf.ctypes.data, ctypes.byref(ts)) == N.MR_ERR_INVALID
    assert lib.mr_toeplitz_image(None, 1024, 100, N.MR_F16, buf.ctypes.data, ctypes.byref(ts)) == N.MR_ERR_INVALID


def split_block_filter(x, g, n_fft, cols, fmt):
    """The kernel's contraction in NumPy: per-row power-of-two input scale, split 16-bit
    parts, x_hi g_hi + near-diagonal cross terms, float64 sums (the GPU sums in FP32)."""
    rnd = f16 if fmt == N.MR_F16 else bf16
    kb = (cols + 63) // 64
    n = 64 * kb
    xp = np.zeros((x.shape[0], n))
    xp[:, :cols] = x
    rs = 2.0 ** (14 - np.frexp(np.abs(xp).max(axis=1, keepdims=True))[1])
    xs = xp * rs
    x_hi = rnd(xs)
    x_lo = rnd(xs - x_hi)
    T = g[(np.arange(n)[:, None] - np.arange(n)[None, :]) % n_fft]
    ts = 2.0 ** (14 - np.frexp(np.abs(g).max())[1])
    T_hi = rnd(T * ts)
    T_lo = rnd(T * ts - T_hi)
    near = np.abs(np.arange(n)[:, None] // 64 - np.arange(n)[None, :] // 64) <= 1
    y = x_hi @ T_hi.T + x_hi @ (T_lo * near).T + x_lo @ (T_hi * near).T
    return (y / ts / rs)[:, :cols]


def smooth_rows(cols, rng):
    c = np.arange(cols)
    return np.array([np.clip(1 - ((c - 240.0) / 180) ** 2, 0, None) * 3 + rng.normal(0, 0.02, cols)
                     for _ in range(6)])


@pytest.mark.parametrize("window", ["ram-lak", "shepp-logan", "hann", "cosine"])
def test_split_fp16_scheme_matches_the_fft_filter(window):
    cols = 486
    g, n_fft = tables(cols, window)
    x = smooth_rows(cols, np.random.default_rng(1))
    want = of.filter_rows(x[None], 1.0, window, exact64=True)[0]
    for scale in (1.0, 1e-6, 1e4):                     # per-row scaling keeps any range
        got = split_block_filter(x * scale, g, n_fft, cols, N.MR_F16) / scale
        assert np.linalg.norm(got - want) / np.linalg.norm(want) < 3e-5


def test_split_bf16_is_limited_by_cancellation():
    """Why FP16 parts are the default: with BF16 parts the same scheme misses the FP64
    filter by ~5e-4 on smooth rows (16 carried bits against ~400x cancellation)."""
    cols = 486
    g, n_fft = tables(cols, "shepp-logan")
    x = smooth_rows(cols, np.random.default_rng(1))
    want = of.filter_rows(x[None], 1.0, "shepp-logan", exact64=True)[0]
    err = lambda fmt: np.linalg.norm(split_block_filter(x, g, n_fft, cols, fmt) - want) / np.linalg.norm(want)  # noqa: E731
    e16, eb16 = err(N.MR_F16), err(N.MR_BF16)
    assert e16 < 3e-5 and 1e-4 < eb16 < 2e-3 and eb16 > 20 * e16
