"""Tensor-core Toeplitz filter (mr_ingest_u16_tc, mr_filter_f32_tc) against the FP64
oracle of the reference's correction + FDK filter (flexray.py:174-184, recon.py:85-104).
Bars: split FP16 operands with an FP32 ring, rel-L2 <= 3e-5 of the FP64 filter; BF16
ring, <= 4e-3 (the store's own rounding, as for the FFT path); split BF16 operands,
<= 2e-3 (their 16 carried bits against the ramp filter's cancellation). Sizes cover one
to eight 64-column blocks, rows that straddle 128-row tiles and views, odd widths (no
vector loads), binning, row flips and caller pitches wider than the accumulator."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import filter as of
from oracle import geometry as og
from tomography_local_demo_b200 import SliceReconstructor, circular_cone_vectors
from tomography_local_demo_b200 import _native as N
from tomography_local_demo_b200 import recon as R

pytestmark = pytest.mark.gpu


def _raw_case(rng, k, rows, cols, bin_):
    R0, C0 = (rows * bin_ + 1, cols * bin_ + 1) if bin_ > 1 else (rows, cols)
    flat = rng.normal(50000, 1000, (2, R0, C0)).clip(0, 65535).astype(np.uint16)
    dark = rng.normal(100, 5, (2, R0, C0)).clip(0, 65535).astype(np.uint16)
    yy, xx = np.mgrid[0:R0, 0:C0]
    atten = np.stack([2.0 * np.exp(-(((xx - C0 * (0.3 + 0.05 * v)) / (0.2 * C0)) ** 2 + ((yy - R0 / 2) / (0.3 * R0)) ** 2))
                      for v in range(k)])
    raw = (rng.poisson((50000 - 100) * np.exp(-atten)) + 100).clip(0, 65535).astype(np.uint16)
    raw[0, 0, 0] = 0                                     # clip at 1e-3
    return raw, flat, dark


def _ingest_tc(raw, d_b, g_b, bin_, flip, K, rows, cols, window, store, fmt, extra_pitch=0):
    dev = torch.device("cuda", 0)
    tables = R._FilterTables(cols, window, dev)
    img, t_scale = tables.tc_image(fmt)
    k = raw.shape[0]
    code, tdt = {"fp32": (N.MR_F32, torch.float32), "bf16": (N.MR_BF16, torch.bfloat16)}[store]
    pitch = (cols + 7) // 8 * 8 + extra_pitch
    ring = torch.full((k + 1, rows, pitch), 7.0, dtype=tdt, device=dev)
    rc = R._ring_struct(ring, code, N.MR_CONE, rows, cols)
    slots = np.arange(k)[::-1].copy() + 1                 # reversed, slot 0 untouched
    fv = R._struct_tensor(R.cone_filter_views(K, rows, cols, tables.n_fft, slots), dev)
    raw_d = torch.from_numpy(np.ascontiguousarray(raw).view(np.int16).copy()).to(dev)
    d_d = torch.from_numpy(d_b.astype(np.float32)).to(dev)
    g_d = torch.from_numpy(g_b.astype(np.float32)).to(dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    v = R.ctypes_void
    N.check(N.load().mr_ingest_u16_tc(v(raw_d.data_ptr()), raw.shape[1] * raw.shape[2], raw.shape[2], bin_,
                                      int(flip), v(d_d.data_ptr()), v(g_d.data_ptr()), k, v(fv.data_ptr()),
                                      v(img.data_ptr()), fmt, t_scale, tables.n_fft, rc, v(status.data_ptr()),
                                      v(torch.cuda.current_stream().cuda_stream)), "ingest_tc")
    torch.cuda.synchronize()
    assert int(status.item()) == 0, "a bounded device-side wait gave up"
    out = ring.float().cpu().numpy()
    assert np.all(out[0] == 7.0)                          # slots not addressed are untouched
    out = out[slots]
    assert np.all(out[:, :, cols:] == 0)                  # pitch padding is written as zeros
    return out[:, :, :cols]


def _reference(raw, flat, dark, bin_, flip, k, window):
    if flip:
        x_ref, d_b, g_b = of.flexray_correct(raw, dark, flat, bin_)
    else:
        d_b = np.mean([of.bin_mean(f, bin_) for f in dark], axis=0)
        f_b = np.mean([of.bin_mean(f, bin_) for f in flat], axis=0)
        g_b = (1.0 / np.maximum(f_b - d_b, 1.0)).astype(np.float32)
        x_ref = np.stack([-np.log(np.clip((of.bin_mean(im, bin_) - d_b) * g_b, 1e-3, None)) for im in raw])
    V = og.circular_cone_vectors(k, 300.0, 600.0, 1.2)
    want = of.fdk_filter_block(np.transpose(x_ref, (1, 0, 2)).astype(np.float32), of.cone_constants(V), window,
                               exact64=True)
    return want, d_b, g_b, V


CASES = [  # rows, cols, k, bin, flip, extra pitch
    (21, 30, 4, 1, False, 0),          # one block, rows straddle views inside one tile
    (21, 30, 4, 2, True, 0),           # binned, flipped, ragged raw edge
    (384, 486, 3, 1, False, 0),        # the bench's detector: eight blocks, 9 tiles
    (130, 100, 5, 1, True, 16),        # two blocks, tiles straddle views, wide pitch
    (40, 300, 7, 1, False, 0),         # five blocks: a 256 + 64 column accumulator split
    (50, 33, 6, 3, False, 32),         # odd width: scalar loads, pitch past the accumulator
]


@pytest.mark.parametrize("rows,cols,k,bin_,flip,extra", CASES)
def test_tc_ingest_matches_fp64_filter(cuda, rows, cols, k, bin_, flip, extra):
    rng = np.random.default_rng(rows + cols)
    raw, flat, dark = _raw_case(rng, k, rows, cols, bin_)
    want, d_b, g_b, V = _reference(raw, flat, dark, bin_, flip, k, "shepp-logan")
    got = _ingest_tc(raw, d_b, g_b, bin_, flip, R.cone_constants(V), rows, cols, "shepp-logan", "fp32",
                     N.MR_F16, extra)
    assert rel_l2(got, want) < 3e-5


@pytest.mark.parametrize("store,fmt,tol", [("bf16", N.MR_F16, 4e-3), ("fp32", N.MR_BF16, 2e-3)])
def test_tc_ingest_bf16_store_and_bf16_operands(cuda, store, fmt, tol):
    rng = np.random.default_rng(5)
    rows, cols, k = 64, 200, 4
    raw, flat, dark = _raw_case(rng, k, rows, cols, 1)
    want, d_b, g_b, V = _reference(raw, flat, dark, 1, False, k, "ram-lak")
    got = _ingest_tc(raw, d_b, g_b, 1, False, R.cone_constants(V), rows, cols, "ram-lak", store, fmt)
    assert rel_l2(got, want) < tol


def test_tc_entry_points_reject_bad_arguments(cuda):
    dev = torch.device("cuda", 0)
    ring = torch.zeros((2, 8, 600), dtype=torch.float32, device=dev)
    rc = R._ring_struct(ring, N.MR_F32, N.MR_CONE, 8, 600)             # 600 columns: > 512
    fake = R.ctypes_void(ring.data_ptr())
    lib = N.load()
    assert lib.mr_filter_f32_tc(fake, 4800, 600, 1, fake, fake, N.MR_F16, 1.0, 1.0, 2048, rc, None,
                                None) == N.MR_ERR_UNSUPPORTED
    rc = R._ring_struct(ring, N.MR_F32, N.MR_CONE, 8, 500)
    assert lib.mr_filter_f32_tc(fake, 4800, 600, 1, fake, fake, N.MR_F16, 3.0, 1.0, 1024, rc, None,
                                None) == N.MR_ERR_INVALID                 # scale not a power of two
    assert lib.mr_ingest_u16_tc(fake, 4800, 600, 1, 0, fake, fake, 1, fake, fake, N.MR_F32, 1.0, 1024, rc,
                                None, None) == N.MR_ERR_INVALID           # operand format


@pytest.mark.parametrize("filt", ["tc", "tc-bf16"])
def test_reconstructor_with_tc_filter(cuda, filt):
    """SliceReconstructor(filter=...): FP32 blocks through mr_filter_f32_tc (host-computed
    power-of-two input scale) and raw counts through mr_ingest_u16_tc give the same slices
    as the FFT filter, within the operand format's bar."""
    from oracle import phantom as oph
    geom = circular_cone_vectors(60, 300.0, 600.0, 48, 72, 2.0)
    proj = oph.project_cone(oph.Phantom(scale=40.0), geom.vectors, 48, 72)
    req = [dict(origin=(1.0, -2.0, 3.0), normal=(0.3, 0.2, 1.0), n=64),
           dict(origin=(0.0, 0.0, 0.0), normal=(1.0, 0.0, 0.0), n=48)]
    want = SliceReconstructor(proj, geom, verbose=False).reconstruct_planes(req)
    got = SliceReconstructor(proj, geom, verbose=False, filter=filt).reconstruct_planes(req)
    tol = 3e-5 if filt == "tc" else 2e-3
    for a, b in zip(got, want):
        assert rel_l2(a, b) < tol
    # raw counts: the fused ingest against the FFT ingest on the same counts
    rng = np.random.default_rng(3)
    atten = np.transpose(proj, (1, 0, 2)) * (2.5 / proj.max())
    counts = (rng.poisson(49900 * np.exp(-atten)) + 100).clip(0, 65535).astype(np.uint16)
    flat = np.full((48, 72), 50000, np.uint16)
    dark = np.full((48, 72), 100, np.uint16)
    recs = []
    for f in ("fft", filt):
        rec = SliceReconstructor(None, geom, verbose=False, filter=f)
        rec.set_flat_dark(flat, dark)
        rec.add_raw_projections(np.arange(60), counts)
        recs.append(rec)
    torch.cuda.synchronize()
    ring_fft = recs[0]._ring[:, :, :72].float().cpu().numpy()
    ring_tc = recs[1]._ring[:, :, :72].float().cpu().numpy()
    assert rel_l2(ring_tc, ring_fft) < tol
    assert int(recs[1]._status.item()) == 0


def test_tc_filter_option_is_validated(cuda):
    geom = circular_cone_vectors(8, 300.0, 600.0, 8, 600, 1.0)
    with pytest.raises(ValueError):
        SliceReconstructor(None, geom, verbose=False, filter="tc")          # > 512 columns
    with pytest.raises(ValueError):
        SliceReconstructor(None, circular_cone_vectors(8, 300.0, 600.0, 8, 60, 1.0), verbose=False, filter="gemm")
