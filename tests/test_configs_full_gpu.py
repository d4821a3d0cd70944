"""The cone-beam configurations at their full sizes (600 raw uint16 views of 486 x 384 at
0.299 mm, SOD 440 / SDD 680 mm, 40 seeded ellipsoids in a 60 mm sphere, flat ~50000 +/- 2 %,
dark ~100 +/- 5, Poisson noise: the bench scan).

Config 2 (batch FDK): the three seeded oblique 512^2 slices, every in-box pixel, against
the oracle run on the same raw counts - the FP32 ring (FFT and tensor-core filters) within
rel-L2 1e-4 of the oracle with the reference's numerics (float32 correction, float64
filter rounded to float32, float64 back-projection sums), the BF16 ring within 1e-3 of
the FP64 oracle, and zero outside the box mask.

Config 5 (serving): on the config-2 ring, slices of 128^2 .. 1024^2 at zoom 1-8 with COR
offsets, answered by the continuously batched server, are bit-identical to the same
requests reconstructed alone.

Config 4 (calibration): the config-2 scan made with the rotation axis 1.7 px off
(det_shift_u = -1.7, as minirecast selftest.py:89-92) and the detector rotated 0.3 deg
about its normal. The gradient calibration (COR shift and tilt) lands within 0.1 px of the
entropy grid-search optimum (recon.py:498-519, refined on a 0.05 px grid) and within
0.1 deg of the baked-in tilt (the entropy criterion itself peaks 0.05-0.08 deg away from
the true tilt on this phantom, measured with the CPU oracle on a grid of shifts and
tilts); the adjoint and geometry gradients pass the dot-product and
central-difference (h = 1e-2 px, 1e-3 deg) checks on a 512^2 slice of this geometry.
"""
import math

import numpy as np
import pytest
import torch

import bench
from conftest import rel_l2
from tomography_local_demo_b200 import ConeVecGeometry, SliceReconstructor, circular_cone_vectors
from tomography_local_demo_b200 import phantom as PH
from tomography_local_demo_b200.server import SliceServer

pytestmark = pytest.mark.gpu

W = bench.WORKLOAD
V, ROWS, COLS = W["views"], W["rows"], W["cols"]


@pytest.fixture(scope="module")
def scan(cuda):
    geom, raw, flats, darks = bench.make_scan(cuda)
    yield geom, raw, bench.as_u16(flats), bench.as_u16(darks)
    del raw
    torch.cuda.empty_cache()


def _ring(geom, raw, flats, darks, store, filt):
    rec = SliceReconstructor(None, geom, store=store, filter=filt, verbose=False)
    rec.set_flat_dark(flats, darks)
    rec.add_raw_projections(np.arange(V), raw)
    return rec


# ------------------------------------------------------------------ config 2
def test_config2_full_size_parity(scan):
    geom, raw, flats, darks = scan
    box = geom.volume_box()
    reqs = bench.slice_requests(box)
    raw_h = raw.cpu().numpy().view(np.uint16)
    ref, _ = bench.cpu_job(raw_h, flats, darks, geom, reqs, box, "ref")
    exact, _ = bench.cpu_job(raw_h, flats, darks, geom, reqs, box, "fp64")
    cases = [("fp32", "fft", ref, 1e-4), ("fp32", "tc", ref, 1e-4), ("bf16", "tc", exact, 1e-3),
             ("bf16", "fft", exact, 1e-3)]
    for store, filt, want, bound in cases:
        rec = _ring(geom, raw, flats, darks, store, filt)
        imgs = rec.reconstruct_planes(reqs)
        for r, (img, (sel, v)) in enumerate(zip(imgs, want)):
            assert not img[~sel].any(), (store, filt, r)           # zero outside the box mask
            assert np.count_nonzero(img[sel]) >= 0.999 * sel.sum(), (store, filt, r)
            err = rel_l2(img[sel], v)
            assert err < bound, (store, filt, r, err)
            print(f"\n[config 2] {store} ring, {filt} filter, slice {r}: {int(sel.sum())} pixels, "
                  f"rel-L2 {err:.2e} (bound {bound:.0e})", end="")
        del rec
    torch.cuda.empty_cache()


# ------------------------------------------------------------------ config 5
def test_config5_alone_and_in_the_mix_on_the_config2_ring(scan):
    geom, raw, flats, darks = scan
    rec = _ring(geom, raw, flats, darks, "bf16", "tc")
    rng = np.random.default_rng(55)
    reqs = []
    for n in (128, 256, 512, 1024) * 6:
        nrm = rng.normal(size=3)
        reqs.append(dict(origin=tuple(rng.uniform(-10, 10, 3)), normal=tuple(nrm / np.linalg.norm(nrm)), n=n,
                         zoom=float(rng.uniform(1, 8)), cor_shift=float(rng.uniform(-10, 10))))
    order = rng.permutation(len(reqs))
    srv = SliceServer(rec, budget_bytes=20e9, max_batch=16, pool_bytes=1 << 30)
    try:
        futs = [srv.submit(**reqs[i]) for i in order]
        mixed = {int(i): f.result(timeout=120) for i, f in zip(order, futs)}
        srv.device_status()
    finally:
        srv.close()
    assert srv.batches >= 2
    for i, r in enumerate(reqs):
        alone = rec.reconstruct_planes_tensor([r])[0].cpu().numpy()
        assert np.count_nonzero(alone) > 0
        np.testing.assert_array_equal(mixed[i], alone)


# ------------------------------------------------------------------ config 4
SHIFT_TRUE, TILT_TRUE_DEG = 1.7, 0.3


def calibration_scan(dev):
    """Raw counts of the bench phantom seen with the rotation axis SHIFT_TRUE px off and
    the detector rotated TILT_TRUE_DEG about its normal (u' = c u + s v, v' = -s u + c v),
    and the nominal geometry that the reconstruction assumes."""
    nominal = bench.geometry()
    vec = circular_cone_vectors(V, W["sod"], W["sdd"], ROWS, COLS, W["pixel"], det_shift_u=-SHIFT_TRUE).vectors.copy()
    t = math.radians(TILT_TRUE_DEG)
    u, v = vec[:, 6:9].copy(), vec[:, 9:12].copy()
    vec[:, 6:9] = math.cos(t) * u + math.sin(t) * v
    vec[:, 9:12] = -math.sin(t) * u + math.cos(t) * v
    ph = PH.EllipsoidPhantom(1.0, PH.random_ellipsoids(W["ellipsoids"], W["phantom_seed"]))
    p = PH.project_cone_torch(ph, ConeVecGeometry(vec, ROWS, COLS), device=dev)
    flat = torch.full((ROWS, COLS), 50000.0, dtype=torch.float64, device=dev)
    dark = torch.full((ROWS, COLS), 100.0, dtype=torch.float64, device=dev)
    raw = PH.raw_counts(p, flat, dark, seed=9).to(torch.int16)
    frames = lambda x: np.full((2, ROWS, COLS), x, np.uint16)       # noqa: E731
    return nominal, raw, frames(50000), frames(100)


def test_config4_gradient_calibration_with_tilt(cuda):
    geom, raw, flats, darks = calibration_scan(cuda)
    rec = _ring(geom, raw, flats, darks, "fp32", "fft")
    coarse, _ = rec.estimate_cor(verbose=False)
    fine_shifts = np.arange(coarse - 0.3, coarse + 0.301, 0.05)
    fine = float(fine_shifts[np.argmax(rec.cor_scores(fine_shifts))])
    shift, tilt, hist = rec.calibrate(shift0=0.0, tilt0=0.0, fit_tilt=True)
    print(f"\n[config 4] grid search {coarse:+.2f} -> {fine:+.2f} px; gradient calibration "
          f"{shift:+.3f} px, {tilt:+.4f} deg in {len(hist) - 1} steps")
    assert abs(shift - fine) <= 0.1, (shift, fine, hist[-3:])
    assert abs(shift - SHIFT_TRUE) <= 0.25, shift
    assert abs(tilt - TILT_TRUE_DEG) <= 0.1, (tilt, hist[-3:])


def test_config4_adjoint_and_gradients_at_full_size(cuda):
    """<B q, y> = <q, B^T y> on a 512^2 oblique slice of the full-size geometry with random
    q, y; the geometry gradients against central differences of a float64 torch
    evaluation of the same operator (smooth q and y as in the small-case test, q windowed
    to 0 at the detector edges)."""
    from test_autograd_gpu import smooth_field, torch64_reference
    from tomography_local_demo_b200 import _native as N
    from tomography_local_demo_b200 import recon as R
    from tomography_local_demo_b200.autograd import BackprojectOp
    geom = bench.geometry()
    grids = np.zeros(1, N.GRID_DTYPE)
    grids[0] = R.plane_grid(geom.volume_box(), (3.0, -2.0, 4.0), (0.3, 0.2, 1.0), 512, None, 1.0, None, 0.0)
    maps = R.cone_view_maps(R.cone_constants(geom.vectors), ROWS, COLS)
    op = BackprojectOp(torch.from_numpy(maps.view(np.uint8).copy()).to(cuda), N.MR_CONE, ROWS, COLS, grids,
                       512 * 512)
    g = torch.Generator(device=cuda).manual_seed(21)
    q = torch.randn((V, ROWS, COLS), generator=g, device=cuda)
    y = torch.rand(op.n_out, generator=g, device=cuda)
    for shift, tilt in ((0.0, 0.0), (1.7, math.radians(0.3))):
        Bq = op.forward(q, shift, tilt)
        BTy = op.adjoint(y, shift, tilt, tuple(q.shape))
        lhs = float((Bq.double() * y.double()).sum())
        rhs = float((q.double() * BTy.double()).sum())
        assert abs(lhs - rhs) <= 1e-5 * max(abs(lhs), abs(rhs)), (shift, tilt, lhs, rhs)
    # finite differences on every 10th view (the float64 reference loops over views)
    sub = np.arange(0, V, 10)
    maps = R.cone_view_maps(R.cone_constants(geom.vectors[sub]), ROWS, COLS)
    qs, ys = smooth_field(len(sub), ROWS, COLS, op.n_out)
    # taps outside the detector read 0, so the operator has a kink wherever a sample crosses
    # the detector edge; at this size those kinks no longer average out of a +/-h difference
    # unless q itself goes to 0 at the edges (a window that vanishes one pixel outside them)
    win = lambda n: torch.sin(math.pi * (torch.arange(n, device=cuda, dtype=torch.float64) + 1) / (n + 1))  # noqa
    qs = (qs.double() * win(ROWS)[None, :, None] * win(COLS)[None, None, :]).float().contiguous()
    op_s = BackprojectOp(torch.from_numpy(maps.view(np.uint8).copy()).to(cuda), N.MR_CONE, ROWS, COLS, grids,
                         512 * 512)
    grids = op_s.grids_at(0.0, 0.0)
    q64 = qs.double()

    def L(s, t):
        f = torch64_reference(q64, maps, grids, torch.tensor(s, dtype=torch.float64, device=cuda),
                              torch.tensor(t, dtype=torch.float64, device=cuda), ROWS, COLS)
        return float((f * ys).sum())

    for s0, t0 in ((0.4, 0.0), (1.7, math.radians(0.3))):
        ds, dt = op_s.grad_geometry(qs, ys.float(), s0, t0)
        h, ht = 1e-2, math.radians(1e-3)
        fd_s = (L(s0 + h, t0) - L(s0 - h, t0)) / (2 * h)
        fd_t = (L(s0, t0 + ht) - L(s0, t0 - ht)) / (2 * ht)
        assert abs(float(ds) - fd_s) <= 1e-2 * abs(fd_s) + 1e-6, (s0, float(ds), fd_s)
        assert abs(float(dt) - fd_t) <= 1e-2 * abs(fd_t) + 1e-6, (s0, float(dt), fd_t)
