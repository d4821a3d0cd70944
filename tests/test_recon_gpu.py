"""SliceReconstructor end to end on the GPU against the reference's own outputs
(golden fixtures from minirecast) and ports of minirecast selftest.py.
Bar: rel-L2 <= 1e-4 for the FP32 store against the reference's Numba path; zero
pattern (box mask) identical; BF16 store rel-L2 <= 1e-3 against the FP64 oracle."""
import numpy as np
import pytest

from conftest import golden, rel_l2
from oracle import phantom as oph
from oracle.recon import OracleReconstructor
from tomography_local_demo_b200 import ConeVecGeometry, ParallelGeometry, SliceReconstructor
from tomography_local_demo_b200 import circular_cone_vectors
from tomography_local_demo_b200.stream import Feeder, arrival_order

pytestmark = pytest.mark.gpu
PH = oph.Phantom(scale=50.0)


def _geom(g, name):
    if name == "cone":
        return ConeVecGeometry(g["V"], int(g["rows"]), int(g["cols"]))
    return ParallelGeometry(g["angles"], int(g["rows"]), int(g["cols"]), 3.5, 4.4)


def same(img, want, mask=None, tol=1e-4):
    """rel-L2 <= tol, and exactly 0 outside the box mask (the reference's mask, FP64).
    Inside the box a value can be exactly 0 in FP64 when every tap misses the detector
    while FP32 coordinates put a tap a hair inside, so zeros are compared on the mask."""
    assert img.shape == want.shape
    if mask is not None:
        assert np.all(img[~mask] == 0) and np.all(want[~mask] == 0)
    assert rel_l2(img, want) < tol


def mask_of(rec, *args, **kw):
    from oracle import geometry as og
    return og.slice_points(rec.box, *args, **kw)[1]


@pytest.mark.parametrize("name", ["cone", "parallel"])
def test_reconstructor_matches_reference_outputs(cuda, name):
    g = golden(f"recon_{name}.npz")
    geom = _geom(g, name)
    rec = SliceReconstructor(g["proj"], geom, verbose=False)
    assert rec.n == geom.n_angles and rec.backend == "cuda-sm100a"
    np.testing.assert_allclose(rec.box, g["box"])
    img, pts = rec.reconstruct_plane((3.0, -2.0, 5.0), (1.0, 0.5, 0.8), n=40, size=110)
    assert pts.shape == (40, 40, 3) and img.dtype == np.float64
    same(img, g["img_oblique"], mask_of(rec, (3.0, -2.0, 5.0), (1.0, 0.5, 0.8), 40, 110))
    img, _ = rec.reconstruct_plane((0, 0, 1.0), (0.3, 0.0, 1.0), n=33, zoom=1.5, center=(2.0, 0, 0),
                                   cor_shift=0.8)
    zmask = mask_of(rec, (0, 0, 1.0), (0.3, 0.0, 1.0), 33, None, 1.5, (2.0, 0, 0))
    same(img, g["img_zoom"], zmask)
    img, _ = rec.reconstruct_plane((0, 0, 0), (0, 0, 1), n=24)
    same(img, g["img_axial"], mask_of(rec, (0, 0, 0), (0, 0, 1), 24))
    vol, origin, h = rec.reconstruct_volume(voxel=8.0)
    assert vol.dtype == np.float32 and vol.shape == g["vol"].shape
    np.testing.assert_allclose(origin, g["vol_origin"])
    assert rel_l2(vol, g["vol"]) < 1e-4
    best, scores = rec.estimate_cor(np.arange(-2.0, 2.01, 0.5), n=32, verbose=False)
    assert best == float(g["cor_best"]) and rec.cor_shift == best
    np.testing.assert_allclose(scores, g["cor_scores"], rtol=2e-3)
    # live streaming in interleaved order, groups of 7
    live = SliceReconstructor(None, geom, verbose=False)
    order = arrival_order(geom.n_angles, "interleaved")
    for i in range(0, len(order), 7):
        live.add_projections(order[i:i + 7], g["proj"][:, order[i:i + 7], :])
    np.testing.assert_array_equal(live._order[:live.n], g["live_order"])
    img, _ = live.reconstruct_plane((0, 0, 1.0), (0.3, 0.0, 1.0), n=33, zoom=1.5, center=(2.0, 0, 0),
                                    cor_shift=0.8)
    same(img, g["img_live"], zmask)


def _selftest_cases():
    pg = ParallelGeometry(np.arange(180) * np.pi / 180, 96, 128, 0.9, 1.15)
    cg = circular_cone_vectors(180, 300.0, 600.0, 128, 160, 1.5, det_shift_u=2.0)
    return [("parallel", pg, oph.project_parallel(PH, pg.angles, 96, 128, 0.9, 1.15)),
            ("cone", cg, oph.project_cone(PH, cg.vectors, 128, 160))]


def _score(img, pts, radius=45.0):
    t = PH.evaluate(pts)
    m = np.linalg.norm(pts, axis=-1) < radius
    return np.median(np.abs(img[m] - t[m])), np.corrcoef(img[m], t[m])[0, 1]


@pytest.fixture(scope="module")
def selftest_data():
    return _selftest_cases()


def test_selftest_accuracy_and_oracle_parity(cuda, selftest_data):
    """selftest.py:37-57: oblique slice vs the phantom (median < 0.01, corr > 0.85) and
    the GPU result against the reference numerics (oracle) on the same data."""
    for name, geom, proj in selftest_data:
        rec = SliceReconstructor(proj, geom, verbose=False)
        rec.warmup()
        img, pts = rec.reconstruct_plane((3.0, -2.0, 5.0), (1.0, 0.5, 0.8), n=128, size=110)
        med, corr = _score(img, pts)
        assert med < 0.01 and corr > 0.85, (name, med, corr)
        ref = OracleReconstructor(proj, geom)
        want, _ = ref.reconstruct_plane((3.0, -2.0, 5.0), (1.0, 0.5, 0.8), n=128, size=110)
        same(img, want, mask_of(rec, (3.0, -2.0, 5.0), (1.0, 0.5, 0.8), 128, 110))
        assert np.max(np.abs(img - want)) < 1e-3          # the selftest's numba == numpy bar


def test_selftest_streaming_equals_batch(cuda, selftest_data):
    """selftest.py:60-75: interleaved stream in groups of 17 == batch (max diff < 1e-4)."""
    for name, geom, proj in selftest_data:
        batch = SliceReconstructor(proj, geom, verbose=False)
        live = SliceReconstructor(None, geom, verbose=False)
        Feeder(live, proj, order="interleaved", group=17, rate=0, verbose=False).run()
        a, _ = batch.reconstruct_plane((0, 0, 3.0), (0.2, 0.1, 1.0), n=64)
        b, _ = live.reconstruct_plane((0, 0, 3.0), (0.2, 0.1, 1.0), n=64)
        assert live.n == geom.n_angles
        assert np.max(np.abs(a - b)) < 1e-4
        # duplicates are ignored (recon.py:353-356)
        assert live.add_projections([0, 1], proj[:, [0, 1], :]) == geom.n_angles


def test_selftest_cor_shift(cuda):
    """selftest.py:78-101: a +3 px centre error is found by estimate_cor."""
    true_shift = 3.0
    for name in ("parallel", "cone"):
        if name == "parallel":
            geom = ParallelGeometry(np.arange(180) * np.pi / 180, 32, 160, 0.9, 0.9)
            proj = np.roll(oph.project_parallel(PH, geom.angles, 32, 160, 0.9, 0.9), 3, axis=2)
        else:
            moved = circular_cone_vectors(180, 300.0, 600.0, 32, 160, 1.5, det_shift_u=-true_shift)
            proj = oph.project_cone(PH, moved.vectors, 32, 160)
            geom = circular_cone_vectors(180, 300.0, 600.0, 32, 160, 1.5)
        rec = SliceReconstructor(proj, geom, verbose=False)
        img0, pts = rec.reconstruct_plane((0, 0, 0), (0, 0, 1), n=96, size=110)
        best, _ = rec.estimate_cor(np.arange(-5.0, 5.01, 0.5), n=96, verbose=False)
        img1, _ = rec.reconstruct_plane((0, 0, 0), (0, 0, 1), n=96, size=110)
        assert abs(best - true_shift) <= 0.5
        assert _score(img1, pts)[0] < _score(img0, pts)[0]


def test_volume_equals_points(cuda):
    """selftest.py:181-192: a volume voxel == the same point reconstructed alone."""
    geom = circular_cone_vectors(60, 300.0, 600.0, 48, 64, 3.5)
    rec = SliceReconstructor(oph.project_cone(PH, geom.vectors, 48, 64), geom, verbose=False)
    vol, origin, h = rec.reconstruct_volume(voxel=5.0)
    i, j, k = (np.array(vol.shape) * [0.3, 0.6, 0.5]).astype(int)
    p = origin + h * np.array([i, j, k])
    assert abs(vol[i, j, k] - rec.reconstruct_points(p[None])[0]) < 1e-5
    pv, _, _ = rec.preview_volume(12)
    assert pv.ndim == 3


@pytest.mark.parametrize("store,bound", [("bf16", 1e-3), ("fp16", 2e-4)])
def test_low_precision_store_vs_fp64_oracle(cuda, selftest_data, store, bound):
    name, geom, proj = selftest_data[1]
    rec = SliceReconstructor(proj, geom, verbose=False, store=store)
    img, _ = rec.reconstruct_plane((3.0, -2.0, 5.0), (1.0, 0.5, 0.8), n=128, size=110)
    ref = OracleReconstructor(proj, geom, precision="fp64")
    want, _ = ref.reconstruct_plane((3.0, -2.0, 5.0), (1.0, 0.5, 0.8), n=128, size=110)
    assert rel_l2(img, want) < bound


def test_batched_planes_equal_single_requests(cuda, selftest_data):
    name, geom, proj = selftest_data[1]
    rec = SliceReconstructor(proj, geom, verbose=False)
    reqs = [dict(origin=(0, 0, z), normal=(0.1 * z, 0.3, 1.0), n=n, zoom=zm, cor_shift=s)
            for z, n, zm, s in ((0, 64, 1.0, 0.0), (5, 100, 2.0, 1.5), (-7, 33, 4.0, -2.0))]
    batch = rec.reconstruct_planes(reqs)
    for rq, img in zip(reqs, batch):
        single, _ = rec.reconstruct_plane(rq["origin"], rq["normal"], rq["n"], zoom=rq["zoom"],
                                          cor_shift=rq["cor_shift"])
        np.testing.assert_array_equal(img, single)


def test_errors_match_reference(cuda):
    with pytest.raises(ValueError):
        SliceReconstructor(None, None)

    class NotAGeometry:                 # has what the constructor reads first, like recon.py:312-334
        n_angles, rows, cols = 4, 8, 8

        def volume_box(self):
            return np.ones(3)

    with pytest.raises(TypeError):
        SliceReconstructor(None, NotAGeometry())
    with pytest.raises(AttributeError):             # the reference also fails on volume_box
        SliceReconstructor(None, object())
    geom = circular_cone_vectors(10, 300.0, 600.0, 8, 8, 3.0)
    with pytest.raises(ValueError):
        SliceReconstructor(None, geom, window="bogus")
    rec = SliceReconstructor(None, geom, verbose=False)
    with pytest.raises(ValueError):
        rec.add_projections([0, 1], np.zeros((8, 3, 8), np.float32))
    assert rec.reconstruct_points(np.zeros((5, 3))).tolist() == [0.0] * 5
    img, _ = rec.reconstruct_plane((0, 0, 0), (0, 0, 1), n=16)
    assert np.all(img == 0)


@pytest.mark.parametrize("kind", ["cuda", "pinned", "numpy", "pageable"])
def test_raw_ingest_input_kinds_and_chunked_upload(cuda, kind):
    """add_raw_projections from device counts (one launch) and from host counts (uploaded
    in chunks that overlap the filtering, staged through pinned buffers when pageable):
    every path stores the same ring bit for bit, also when the call repeats views
    (dedup) and when the chunks outnumber the pinned staging buffers."""
    import torch
    geom = circular_cone_vectors(40, 300.0, 600.0, 24, 36, 3.0)
    rng = np.random.default_rng(4)
    raw = rng.integers(2000, 45000, (40, 48, 72)).astype(np.uint16)        # binned 2x2 on ingest
    flat = rng.normal(50000, 500, (2, 48, 72)).clip(0, 65535).astype(np.uint16)
    dark = rng.normal(100, 5, (2, 48, 72)).clip(0, 65535).astype(np.uint16)

    def ingest(src, chunk_bytes):
        rec = SliceReconstructor(None, geom, verbose=False, store="bf16")
        rec.set_flat_dark(flat, dark, bin=2, flip_rows=True)
        rec.upload_chunk_bytes = chunk_bytes
        order = arrival_order(40, "interleaved")
        rec.add_raw_projections(order[:25], src(order[:25]))
        rec.add_raw_projections(order[20:], src(order[20:]))          # 5 repeated views
        torch.cuda.synchronize()
        assert rec.n == 40
        return rec, rec._ring.float().cpu().numpy(), rec._order.copy()

    want_rec, want, want_order = ingest(lambda i: torch.from_numpy(raw[i].view(np.int16)).cuda(), 1 << 30)
    src = {"cuda": lambda i: torch.from_numpy(raw[i].view(np.int16)).cuda(),
           "pinned": lambda i: torch.from_numpy(raw[i].view(np.int16)).pin_memory(),
           "numpy": lambda i: raw[i],
           "pageable": lambda i: torch.from_numpy(raw[i].view(np.int16).copy())}[kind]
    rec, got, order = ingest(src, 3 * 48 * 72 * 2)                         # 3 views per chunk
    np.testing.assert_array_equal(order, want_order)
    np.testing.assert_array_equal(got, want)
    # right after a chunked host upload a slice sums the views chunk by chunk (each partial
    # launch waits only for its chunk): the same result up to the FP32 summation order
    req = dict(origin=(1.0, -2.0, 0.5), normal=(0.3, 0.2, 1.0), n=40)
    got_img = rec.reconstruct_planes([req])[0]
    want_img = want_rec.reconstruct_planes([req])[0]
    np.testing.assert_array_equal(got_img == 0, want_img == 0)
    assert rel_l2(got_img, want_img) < 1e-6
    if kind != "cuda":
        assert len(rec._chunk_marks) >= 2            # the split path was taken


@pytest.mark.gpu
def test_reset_reuses_resident_records(cuda):
    """reset() keeps the ring and the view table: a new scan in the same order reuses the
    resident view records, one in another order rewrites them; both reconstruct exactly as
    a fresh reconstructor fed the same way."""
    import torch
    geom = circular_cone_vectors(48, 300.0, 600.0, 24, 36, 3.0)
    rng = np.random.default_rng(8)
    raw = rng.integers(2000, 45000, (48, 24, 36)).astype(np.uint16)
    flat = rng.normal(50000, 500, (2, 24, 36)).clip(0, 65535).astype(np.uint16)
    dark = rng.normal(100, 5, (2, 24, 36)).clip(0, 65535).astype(np.uint16)
    req = [dict(origin=(0.5, -1.0, 0.3), normal=(0.2, 0.3, 1.0), n=40), dict(origin=(0, 0, 0), normal=(1, 0, 0), n=32)]

    def fresh(order):
        rec = SliceReconstructor(None, geom, verbose=False, store="bf16", filter="tc")
        rec.set_flat_dark(flat, dark)
        for part in np.array_split(order, 3):
            rec.add_raw_projections(part, torch.from_numpy(raw[part].view(np.int16)).cuda())
        return [x.cpu().numpy() for x in rec.reconstruct_planes_tensor(req)]

    def feed(rec, order):
        rec.reset()
        for part in np.array_split(order, 3):
            rec.add_raw_projections(part, torch.from_numpy(raw[part].view(np.int16)).cuda())
        return [x.cpu().numpy() for x in rec.reconstruct_planes_tensor(req)]

    in_order = np.arange(48)
    shuffled = arrival_order(48, "interleaved")
    rec = SliceReconstructor(None, geom, verbose=False, store="bf16", filter="tc")
    rec.set_flat_dark(flat, dark)
    want_a, want_b = fresh(in_order), fresh(shuffled)
    for order, want in ((in_order, want_a), (in_order, want_a), (shuffled, want_b), (in_order, want_a),
                        (shuffled, want_b), (shuffled, want_b)):
        got = feed(rec, order)
        for g, w in zip(got, want):
            np.testing.assert_array_equal(g, w)


@pytest.mark.gpu
def test_empty_calls(cuda):
    """Zero views and zero requests are no-ops on every ingest path."""
    import torch
    geom = circular_cone_vectors(24, 300.0, 600.0, 16, 20, 3.0)
    flat = np.full((1, 16, 20), 40000, np.uint16)
    dark = np.full((1, 16, 20), 100, np.uint16)
    none = np.zeros(0, np.int64)
    for parker in (False, True):
        g = geom if not parker else circular_cone_vectors(24, 300.0, 600.0, 16, 20, 3.0,
                                                          angular_range=np.pi + 0.5)
        rec = SliceReconstructor(None, g, verbose=False, store="bf16", filter="tc", parker=parker)
        rec.set_flat_dark(flat, dark)
        assert rec.add_raw_projections(none, np.zeros((0, 16, 20), np.uint16)) == 0
        assert rec.add_raw_projections(none, torch.zeros((0, 16, 20), dtype=torch.int16).cuda()) == 0
        assert rec.add_projections(none, np.zeros((16, 0, 20), np.float32)) == 0
        assert rec.reconstruct_planes([]) == []
        img, _ = rec.reconstruct_plane((0, 0, 0), (0, 0, 1), n=8)
        assert img.shape == (8, 8) and np.all(img == 0)
