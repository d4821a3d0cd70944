"""The measured configurations at their full sizes, on seeded synthetic scans.

Config 1 (plain parallel-beam FBP, 128^3 Shepp-Logan, 180 views of 128 x 128, Poisson
counts at I0 = 1e4, Shepp-Logan filter, three axis-aligned 128^2 slices): the GPU slices
against the oracle run with the reference's numerics on the same data (rel-L2 <= 1e-4)
and against the FP64 oracle.

Config 3 (full resolution: 1200 uint16 views of 1944 x 1536 at 0.0748 mm, ram-lak, a batch
of 96 slices of 256^2..1024^2 at zoom 1-8, a 640^3 volume at 82.5 um), too large for the
oracle as a whole, checked by properties that hold at any size: the fused raw ingest of
two whole views against the oracle's correction + FDK filter (rel-L2 <= 5e-5: FP32 FFTs of
4096 points on noisy rows under the unwindowed ram-lak filter), the
back-projection of a 60-view slot range of the full-size ring against the oracle on those
views (rel-L2 <= 5e-5), the 96-slice batch equal to the same requests one by one (the
cluster reduction order does not depend on the batch), BF16 against FP32 stacks
(rel-L2 <= 1e-3 per slice), and volume voxels against point requests at their centres
(rel-L2 <= 1e-4: the two paths round the sample coordinates differently).
"""
import time

import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import bp as obp
from oracle import filter as of
from oracle import phantom as oph
from oracle.recon import OracleReconstructor
from tomography_local_demo_b200 import ParallelGeometry, SliceReconstructor, circular_cone_vectors
from tomography_local_demo_b200 import _native as N
from tomography_local_demo_b200 import phantom as PH
from tomography_local_demo_b200 import recon as R

pytestmark = pytest.mark.gpu


# ------------------------------------------------------------------ config 1
def test_config1_parallel_shepp_logan(cuda):
    geom = ParallelGeometry(np.arange(180) * np.pi / 180, 128, 128, 1.0 / 128, 1.0 / 128)
    ph = oph.Phantom(scale=0.5)                              # unit-cube extent
    p = oph.project_parallel(ph, geom.angles, 128, 128, 1.0 / 128, 1.0 / 128)
    counts = np.random.default_rng(0).poisson(1e4 * np.exp(-p.astype(np.float64)))
    proj = (-np.log(np.maximum(counts, 1) / 1e4)).astype(np.float32)
    rec = SliceReconstructor(proj, geom, window="shepp-logan", verbose=False)
    ref = OracleReconstructor(proj, geom, window="shepp-logan", precision="ref")
    f64 = OracleReconstructor(proj, geom, window="shepp-logan", precision="fp64")
    for normal in ((1, 0, 0), (0, 1, 0), (0, 0, 1)):
        img, pts = rec.reconstruct_plane((0, 0, 0), normal, n=128)
        want, _ = ref.reconstruct_plane((0, 0, 0), normal, n=128)
        exact, _ = f64.reconstruct_plane((0, 0, 0), normal, n=128)
        assert np.array_equal(img == 0, want == 0)
        assert rel_l2(img, want) < 1e-4, normal
        assert rel_l2(img, exact) < 1e-4, normal
        # and it is a reconstruction of the phantom
        m = np.abs(ph.evaluate(pts)) > 0
        assert np.corrcoef(img[m], ph.evaluate(pts)[m])[0, 1] > 0.9


# ------------------------------------------------------------------ config 3
VIEWS, ROWS, COLS, PIXEL = 1200, 1536, 1944, 0.0748


def make_full_scan(dev):
    """Raw uint16 counts [1200, 1536, 1944] on the device (flat ~50000 +/- 2 %, dark ~100 +/- 5,
    Poisson) of 40 seeded ellipsoids, plus 4 flat / dark frames, and the geometry."""
    geom = circular_cone_vectors(VIEWS, 440.0, 680.0, ROWS, COLS, PIXEL)
    geom.box = np.array([26.4, 26.4, 26.4])                  # 640 voxels of 82.5 um
    ph = PH.EllipsoidPhantom(1.0, PH.random_ellipsoids(40, 2))
    g = torch.Generator(device=dev)
    g.manual_seed(3)
    flat = 50000.0 * (1.0 + 0.02 * torch.randn((ROWS, COLS), generator=g, device=dev, dtype=torch.float64))
    dark = 100.0 + 5.0 * torch.randn((ROWS, COLS), generator=g, device=dev, dtype=torch.float64)
    raw = torch.empty((VIEWS, ROWS, COLS), dtype=torch.int16, device=dev)
    step = 40
    for k0 in range(0, VIEWS, step):
        sub = type(geom)(geom.vectors[k0:k0 + step], ROWS, COLS)
        p = PH.project_cone_torch(ph, sub, device=dev, views_per_batch=8)
        raw[k0:k0 + step] = PH.raw_counts(p, flat, dark, seed=k0).to(torch.int16)
        del p
    frames = lambda f: torch.stack([f + torch.randn(f.shape, generator=g, device=dev, dtype=torch.float64)  # noqa: E731
                                    for _ in range(4)]).round().clamp(0, 65535).to(torch.int32).cpu().numpy()
    flats, darks = frames(flat).astype(np.uint16), frames(dark).astype(np.uint16)
    return geom, raw, flats, darks


@pytest.fixture(scope="module")
def full_scan():
    scan = make_full_scan(torch.device("cuda", 0))
    yield scan
    del scan
    torch.cuda.empty_cache()


def _ingest(geom, raw, flats, darks, store):
    rec = SliceReconstructor(None, geom, window="ram-lak", store=store, verbose=False)
    rec.set_flat_dark(flats, darks)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rec.add_raw_projections(np.arange(VIEWS), raw)
    torch.cuda.synchronize()
    return rec, time.perf_counter() - t0


def _requests(box):
    rng = np.random.default_rng(96)
    reqs = []
    for _ in range(96):
        nrm = rng.normal(size=3)
        reqs.append(dict(origin=rng.uniform(-10, 10, 3), normal=nrm / np.linalg.norm(nrm),
                         n=int(rng.choice([256, 384, 512, 768, 1024])), zoom=float(rng.uniform(1.0, 8.0))))
    return reqs


def test_config3_full_resolution(cuda, full_scan):
    geom, raw, flats, darks = full_scan
    rec32, t_ingest = _ingest(geom, raw, flats, darks, "fp32")
    print(f"\n[config 3] ingest of {VIEWS} raw views {COLS}x{ROWS} (fp32 ring): {t_ingest * 1e3:.1f} ms")

    # (1) the fused ingest of two whole views against the oracle's correction + FDK filter
    dark_h, gain_h = rec32._dark.cpu().numpy(), rec32._gain.cpu().numpy()
    K = of.cone_constants(geom.vectors)
    for v in (0, 777):
        counts = (raw[v].cpu().numpy().view(np.uint16)).astype(np.float32)
        x = -np.log(np.maximum((counts - dark_h) * gain_h, np.float32(1e-3)))
        want = of.fdk_filter_block(x[:, None, :].astype(np.float32), {k: a[v:v + 1] for k, a in K.items()},
                                   "ram-lak", True)[0]
        got = rec32._ring[v, :, :COLS].cpu().numpy()
        assert rel_l2(got, want) < 5e-5, v

    # (2) back-projection over slots [0, 60) of the full-size ring against the oracle
    rng = np.random.default_rng(5)
    pts = rng.uniform(-20, 20, (3000, 3))
    p_dev = torch.from_numpy(pts.astype(np.float32)).cuda()
    gr = np.zeros(1, N.GRID_DTYPE)
    gr["n_i"], gr["n_j"], gr["n_k"] = 1, len(pts), 1
    gr["flags"] = N.MR_GRID_POINTS
    gr["out_stride_j"] = 1
    gr["points"] = p_dev.data_ptr()
    gr["view_begin"], gr["n_views"], gr["scale"] = 0, 60, np.pi / 60
    out = torch.zeros(len(pts), dtype=torch.float32, device="cuda")
    st = torch.cuda.current_stream()
    R.backproject_device(rec32._ring_c, rec32._views_dev, gr, out, st, out.device, kernel="plain")
    torch.cuda.synchronize()
    q = rec32._ring[:60, :, :COLS].cpu().numpy()
    want = obp.bp_cone(q, K["s"][:60], K["d"][:60], K["uu"][:60], K["vv"][:60], K["n"][:60], K["sdd"][:60],
                       K["sod"][:60], pts, np.pi / 60)
    assert rel_l2(out.cpu().numpy(), want) < 5e-5
    del q

    # (3) 96 slices in one launch = the same requests one by one; BF16 stack vs FP32 stack
    reqs = _requests(geom.box)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    batch32 = rec32.reconstruct_planes_tensor(reqs)
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - t0
    for i in (0, 17, 95):
        one = rec32.reconstruct_planes_tensor([reqs[i]])[0]
        assert torch.equal(one, batch32[i]), i
    imgs32 = [b.cpu().numpy() for b in batch32]
    del batch32
    rec16, _ = _ingest(geom, raw, flats, darks, "bf16")
    imgs16 = [b.cpu().numpy() for b in rec16.reconstruct_planes_tensor(reqs)]
    errs = [rel_l2(b, a) for a, b in zip(imgs32, imgs16) if np.abs(a).max() > 0]
    assert len(errs) > 80 and max(errs) < 1e-3, max(errs)
    print(f"[config 3] 96 slices {t_batch * 1e3:.1f} ms (fp32 stack); bf16 vs fp32 rel-L2 max {max(errs):.2e}")
    del imgs32, imgs16

    # (4) the 640^3 volume at 82.5 um (bf16 stack): voxels = point requests at their centres
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    vol, origin, h = rec16.reconstruct_volume_tensor(voxel=0.0825)
    torch.cuda.synchronize()
    t_vol = time.perf_counter() - t0
    assert tuple(vol.shape) == (640, 640, 640)
    idx = np.random.default_rng(7).integers(0, 640, (2000, 3))
    centres = origin + h * idx
    got = vol[idx[:, 0], idx[:, 1], idx[:, 2]].cpu().numpy()
    want = rec16.reconstruct_points(centres)
    assert rel_l2(got, want) < 1e-4
    print(f"[config 3] 640^3 volume {t_vol * 1e3:.1f} ms = {640 ** 3 * VIEWS / t_vol / 1e9:.0f} G updates/s")
    del vol, rec16, rec32
    torch.cuda.empty_cache()
