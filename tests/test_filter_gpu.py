"""Filter / ingest kernels (mr_filter_f32, mr_ingest_u16, preprocessing) against the
reference's golden vectors and the NumPy oracle. Tolerance: FP32 FFT vs the reference's
float64 (cone) / complex64 (parallel) FFT, max error <= 2e-6 of the output's peak."""
import numpy as np
import pytest
import torch

from conftest import golden, rel_l2
from oracle import filter as of
from tomography_local_demo_b200 import _native as N
from tomography_local_demo_b200 import preprocess as P
from tomography_local_demo_b200 import recon as R

pytestmark = pytest.mark.gpu


def close(got, want, tol=2e-6):
    scale = max(np.abs(want).max(), 1e-30)
    assert np.max(np.abs(np.asarray(got, np.float64) - want)) <= tol * scale


def test_filter_rows_matches_reference(cuda):
    g = golden("filter_rows.npz")
    for w in ("ram-lak", "shepp-logan", "hann", "cosine"):
        close(R.filter_rows(g["x"], 0.9, w), g[f"y_{w}"])


def test_fdk_filter_block_matches_reference(cuda):
    g = golden("fdk.npz")
    K = R.cone_constants(g["V_gen"])
    for w in ("shepp-logan", "ram-lak"):
        close(R.fdk_filter_block(g["block"], K, w), g[f"fdk_{w}"])


@pytest.mark.parametrize("cols", [5, 9, 20, 33, 64, 128, 200, 486, 1000, 1944, 4000])
def test_filter_rows_all_fft_lengths(cuda, cols):
    rng = np.random.default_rng(cols)
    x = rng.normal(0, 1, (5, 3, cols)).astype(np.float32)     # odd row count per view
    want = of.filter_rows(x, 0.37, "shepp-logan", exact64=True)
    got = R.filter_rows(x, 0.37, "shepp-logan")
    assert rel_l2(got, want) < 1e-6
    close(got, want, 3e-6)


def test_fdk_cone_case_size(cuda):
    from oracle import geometry as og
    rng = np.random.default_rng(0)
    V = og.circular_cone_vectors(6, 440.0, 680.0, 0.299)
    K = of.cone_constants(V)
    block = rng.normal(1, 0.5, (384, 6, 486)).astype(np.float32)
    want = of.fdk_filter_block(block, K, "shepp-logan", exact64=True)
    got = R.fdk_filter_block(block, R.cone_constants(V), "shepp-logan")
    assert rel_l2(got, want) < 1e-6


def _ingest(raw, dark, gain, bin_, flip, K, rows, cols, window, store="fp32"):
    dev = torch.device("cuda", 0)
    tables = R._FilterTables(cols, window, dev)
    k = raw.shape[0]
    code, tdt = {"fp32": (N.MR_F32, torch.float32), "bf16": (N.MR_BF16, torch.bfloat16)}[store]
    pitch = (cols + 7) // 8 * 8
    ring = torch.full((k, rows, pitch), 7.0, dtype=tdt, device=dev)
    rc = R._ring_struct(ring, code, N.MR_CONE, rows, cols)
    fv = R._struct_tensor(R.cone_filter_views(K, rows, cols, tables.n_fft, np.arange(k)), dev)
    raw_d = torch.from_numpy(np.ascontiguousarray(raw).view(np.int16).copy()).to(dev)   # uint16 bits
    d_d = torch.from_numpy(dark.astype(np.float32)).to(dev)
    g_d = torch.from_numpy(gain.astype(np.float32)).to(dev)
    st = torch.cuda.current_stream()
    v = R.ctypes_void
    N.check(N.load().mr_ingest_u16(v(raw_d.data_ptr()), raw.shape[1] * raw.shape[2], raw.shape[2], bin_,
                                   int(flip), v(d_d.data_ptr()), v(g_d.data_ptr()), k,
                                   v(fv.data_ptr()), v(tables.H.data_ptr()), v(tables.tw.data_ptr()),
                                   tables.log2n, rc, v(st.cuda_stream)), "ingest")
    torch.cuda.synchronize()
    out = ring.float().cpu().numpy()
    assert np.all(out[:, :, cols:] == 0)          # pitch padding is written as zeros
    return out[:, :, :cols]


@pytest.mark.parametrize("bin_,flip", [(1, False), (2, True), (3, False)])
def test_raw_ingest_matches_flexray_correction_plus_fdk(cuda, bin_, flip):
    from oracle import geometry as og
    rng = np.random.default_rng(bin_)
    rows, cols, k = 21, 30, 4
    # binned readers crop a ragged raw edge; sample 1 reads the frame as it is
    R0, C0 = (rows * bin_ + 1, cols * bin_ + 1) if bin_ > 1 else (rows, cols)
    flat = rng.normal(50000, 1000, (2, R0, C0)).clip(0, 65535).astype(np.uint16)
    dark = rng.normal(100, 5, (2, R0, C0)).clip(0, 65535).astype(np.uint16)
    atten = rng.uniform(0.05, 3.0, (k, R0, C0))
    raw = (rng.poisson((50000 - 100) * np.exp(-atten)) + 100).clip(0, 65535).astype(np.uint16)
    raw[0, 0, 0] = 0                                                     # clip at 1e-3 path
    if flip:
        x_ref, d_b, g_b = of.flexray_correct(raw, dark, flat, bin_)
    else:
        def binned(a):
            return of.bin_mean(a, bin_)
        d_b = np.mean([binned(f) for f in dark], axis=0)
        f_b = np.mean([binned(f) for f in flat], axis=0)
        g_b = (1.0 / np.maximum(f_b - d_b, 1.0)).astype(np.float32)
        x_ref = np.stack([-np.log(np.clip((binned(im) - d_b) * g_b, 1e-3, None)) for im in raw])
    V = og.circular_cone_vectors(k, 300.0, 600.0, 1.2)
    K = of.cone_constants(V)
    want = of.fdk_filter_block(np.transpose(x_ref, (1, 0, 2)).astype(np.float32), K, "hann", exact64=True)
    got = _ingest(raw, d_b, g_b, bin_, flip, R.cone_constants(V), rows, cols, "hann")
    assert rel_l2(got, want) < 2e-6


@pytest.mark.parametrize("cols,flip", [(700, False), (1944, True), (2040, False)])
def test_raw_ingest_wide_rows(cuda, cols, flip):
    """2048- and 4096-point rows: the ingest keeps each CTA on one row pair with the pair's
    dark / gain rows in shared memory next to float exchange buffers; at 2040 columns those
    no longer fit beside two CTAs an SM and the CTAs stride over all items. Odd row count
    (the last pair has one row), more views than one CTA's slots, per-pixel fields."""
    from oracle import geometry as og
    rng = np.random.default_rng(cols)
    rows, k = 5, 37
    d_b = rng.normal(100, 5, (rows, cols)).astype(np.float32)
    g_b = (1.0 / rng.normal(49900, 800, (rows, cols))).astype(np.float32)
    atten = rng.uniform(0.05, 3.0, (k, rows, cols))
    raw = (rng.poisson(49900 * np.exp(-atten)) + 100).clip(0, 65535).astype(np.uint16)
    # a flipped read takes the frame's rows bottom-up; dark / gain are given in output order
    src = raw[:, ::-1, :] if flip else raw
    d_f, g_f = (d_b[::-1].copy(), g_b[::-1].copy()) if flip else (d_b, g_b)
    x = -np.log(np.clip((src.astype(np.float32) - d_f) * g_f, 1e-3, None))
    V = og.circular_cone_vectors(k, 440.0, 680.0, 0.0748 * 1944 / cols)
    want = of.fdk_filter_block(np.transpose(x, (1, 0, 2)).astype(np.float32), of.cone_constants(V), "ram-lak",
                               exact64=True)
    got = _ingest(raw, d_f, g_f, 1, flip, R.cone_constants(V), rows, cols, "ram-lak")
    assert rel_l2(got, want) < 2e-6


def test_raw_ingest_bf16_store(cuda):
    from oracle import geometry as og
    rng = np.random.default_rng(0)
    rows, cols, k = 16, 40, 3
    raw = rng.integers(3000, 40000, (k, rows, cols)).astype(np.uint16)
    d_b = np.full((rows, cols), 100.0, np.float32)
    g_b = np.full((rows, cols), 1.0 / 49900.0, np.float32)
    V = og.circular_cone_vectors(k, 300.0, 600.0, 1.2)
    x = -np.log(np.clip((raw.astype(np.float32) - d_b) * g_b, 1e-3, None))
    want = of.fdk_filter_block(np.transpose(x, (1, 0, 2)), of.cone_constants(V), "ram-lak", exact64=True)
    got = _ingest(raw, d_b, g_b, 1, False, R.cone_constants(V), rows, cols, "ram-lak", "bf16")
    assert rel_l2(got, want) < 4e-3


@pytest.mark.parametrize("op", ["gauss", "rot", "apply"])
def test_preprocess_matches_reference(cuda, op):
    g = golden("preprocess.npz")
    if op == "gauss":
        close(P.gaussian_blur(g["block"], 1.5), g["gauss_1_5"], 1e-5)
    elif op == "rot":
        close(P.rotate_projections(g["block"], 7.0), g["rot_7"], 1e-5)
    else:
        close(P.apply(g["block"], gaussian=0.8, tilt=2.5), g["apply"], 1e-5)
    rot = P.rotate_projections(g["point"], 90.0)
    r, c = np.unravel_index(np.argmax(rot[:, 0, :]), (41, 41))
    assert (r, c) in ((10, 20), (30, 20))


@pytest.mark.parametrize("shape,sigma", [((96, 7, 150), 1.0), ((37, 5, 300), 0.8), ((130, 3, 61), 2.5),
                                         ((384, 2, 486), 1.0)])
def test_gaussian_blur_against_oracle_at_size(cuda, shape, sigma):
    """The staged shared-memory Gaussian (lines that are not a multiple of the block's line
    count, lengths that are not a multiple of its output span, taps reaching half the
    padded length at small sigma) against the oracle's FFT restatement of
    preprocess.py:8-28."""
    rng = np.random.default_rng(int(sigma * 10) + shape[0])
    block = rng.normal(1.0, 0.3, shape).astype(np.float32)
    close(P.gaussian_blur(block, sigma), of.gaussian_blur(block, sigma), 1e-5)
