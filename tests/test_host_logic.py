"""Host-side logic of the product (no GPU): FP64 geometry, projective maps, filter
parameters, plane/volume grid records and the tile planner, against the oracle and the
reference's golden vectors."""
import numpy as np
import pytest

from conftest import golden
from oracle import filter as of
from oracle import geometry as og
from tomography_local_demo_b200 import _native as N
from tomography_local_demo_b200 import geometry as G
from tomography_local_demo_b200 import recon as R
from tomography_local_demo_b200 import stream as S


def test_ramp_response_matches_reference():
    g = golden("ramp.npz")
    for key, H in g.items():
        _, n, tau, w = key.split("_", 3)
        Hp, N_ = R.ramp_response(int(n), float(tau), w)
        assert N_ == len(H)
        np.testing.assert_allclose(Hp, H, rtol=0, atol=1e-12 * np.abs(H).max())
    with pytest.raises(ValueError):
        R.ramp_response(16, 1.0, "bogus")


def test_geometry_containers_match_reference():
    g = golden("phantom.npz")
    cg = G.circular_cone_vectors(9, 300.0, 600.0, 10, 12, 15.0, det_shift_u=1.5)
    np.testing.assert_allclose(cg.vectors, g["cone_V"], rtol=1e-15, atol=1e-12)
    np.testing.assert_allclose(cg.volume_box(), og.cone_volume_box(cg.vectors, 10, 12), rtol=1e-15)
    pg = G.ParallelGeometry(np.arange(9) * np.pi / 9, 10, 12, 9.0, 11.0)
    np.testing.assert_allclose(pg.volume_box(), og.parallel_volume_box(10, 12, 9.0, 11.0))
    assert pg.n_angles == 9 and cg.n_angles == 9
    fg = golden("fdk.npz")
    K = R.cone_constants(fg["V_gen"])
    for k in K:
        np.testing.assert_allclose(K[k], fg["K_" + k], rtol=1e-14, atol=1e-12)


def _ref_project(K, k, p, rows, cols, shift=0.0):
    """recon.py:206-217 in float64 for one view and points p [M,3]."""
    D = K["d"][k] - shift * K["u"][k]
    rel = p - K["s"][k]
    L = rel @ K["n"][k]
    t = K["sdd"][k] / L
    X = K["s"][k] + t[:, None] * rel - D
    return (X @ K["vv"][k] + (rows - 1) / 2.0, X @ K["uu"][k] + (cols - 1) / 2.0,
            (K["sod"][k] / L) ** 2)


@pytest.mark.parametrize("shift", [0.0, 1.7, -3.2])
def test_cone_view_maps_reproduce_reference_projection(shift):
    fg = golden("fdk.npz")
    V = fg["V_gen"]
    rows, cols = 16, 20
    K = R.cone_constants(V)
    maps = R.cone_view_maps(K, rows, cols)
    rng = np.random.default_rng(3)
    p = rng.uniform(-20, 20, (50, 3))
    ph = np.concatenate([p, np.ones((50, 1))], 1)
    for k in range(len(V)):
        pu = maps["pu"][k].astype(np.float64) + shift * maps["pw"][k]
        pv = maps["pv"][k].astype(np.float64) + shift * maps["uv"][k] * maps["pw"][k]
        den = ph @ maps["pw"][k].astype(np.float64)
        row_r, col_r, w_r = _ref_project(K, k, p, rows, cols, shift)
        # FP32-rounded map coefficients: agreement to ~1e-5 detector pixels
        np.testing.assert_allclose((ph @ pu) / den, col_r, atol=2e-4)
        np.testing.assert_allclose((ph @ pv) / den, row_r, atol=2e-4)
        np.testing.assert_allclose(1.0 / den ** 2, w_r, rtol=1e-5)


def test_parallel_view_maps():
    a = np.array([0.0, 0.3, 2.0])
    maps = R.parallel_view_maps(a, 0.9, 1.1, 16, 20)
    p = np.array([[1.0, -2.0, 3.0], [0.5, 0.25, -4.0]])
    ph = np.concatenate([p, np.ones((2, 1))], 1)
    for k in range(3):
        col = (-p[:, 0] * np.sin(a[k]) + p[:, 1] * np.cos(a[k])) / 0.9 + 9.5
        np.testing.assert_allclose(ph @ maps["pu"][k].astype(np.float64), col, atol=1e-5)
        np.testing.assert_allclose(ph @ maps["pv"][k].astype(np.float64), p[:, 2] / 1.1 + 7.5, atol=1e-5)
        assert tuple(maps["pw"][k]) == (0, 0, 0, 1)


def test_cone_filter_views_reproduce_fdk_weight():
    fg = golden("fdk.npz")
    K = R.cone_constants(fg["V_gen"])
    rows, cols = 16, 20
    fv = R.cone_filter_views(K, rows, cols, 64, np.arange(7))
    cc = np.arange(cols) - (cols - 1) / 2.0
    rr = np.arange(rows) - (rows - 1) / 2.0
    for k in range(7):
        s, d, u, v, n = (K[x][k] for x in ("s", "d", "u", "v", "n"))
        sdd, sod = K["sdd"][k], K["sod"][k]
        off = d - (s + sdd * n)
        un, vn = np.linalg.norm(u), np.linalg.norm(v)
        a = off @ u / un + cc * un
        b = off @ v / vn + rr * vn
        w_ref = sdd / np.sqrt(sdd ** 2 + a[None, :] ** 2 + b[:, None] ** 2)
        a2 = fv["a0"][k] + np.arange(cols) * fv["da"][k]
        b2 = fv["b0"][k] + np.arange(rows) * fv["db"][k]
        w2 = fv["sdd"][k] / np.sqrt(fv["sdd"][k] ** 2 + a2[None, :] ** 2 + b2[:, None] ** 2)
        np.testing.assert_allclose(w2, w_ref, rtol=1e-6)
        np.testing.assert_allclose(1.0 / (fv["gain"][k] * 64), un * sod / sdd, rtol=1e-6)


def _device_mask(g):
    """The FP64 mask formula of bp.cu:in_box_fp64, evaluated in NumPy with the same
    operation order (no fused multiply-add)."""
    n_i, n_j = int(g["n_i"]), int(g["n_j"])
    aj = (np.arange(n_j) - g["mask_half"]) * g["mask_delta"]
    ai = (np.arange(n_i) - g["mask_half"]) * g["mask_delta"]
    ok = np.ones((n_i, n_j), bool)
    for e in range(3):
        p = (g["mask_c"][e] + aj[None, :] * g["mask_ej"][e]) + ai[:, None] * g["mask_ei"][e]
        ok &= np.abs(p) <= g["box"][e]
    return ok


@pytest.mark.parametrize("seed", range(6))
def test_plane_grid_mask_and_points_match_slice_points(seed):
    rng = np.random.default_rng(seed)
    box = np.array([47.0, 47.0, 37.2]) * rng.uniform(0.5, 1.5)
    normal = rng.normal(size=3)
    origin = rng.uniform(-10, 10, 3)
    n = int(rng.integers(16, 200))
    zoom = float(rng.uniform(0.5, 3.0))
    center = None if seed % 2 else rng.uniform(-5, 5, 3)
    g = R.plane_grid(box, origin, normal, n, None, zoom, center)
    pts, mask = og.slice_points(box, origin, normal, n, None, zoom, center)
    np.testing.assert_array_equal(_device_mask(g), mask)
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    p32 = (g["origin"].astype(np.float64) + i[..., None] * g["step_i"].astype(np.float64)
           + j[..., None] * g["step_j"].astype(np.float64))
    np.testing.assert_allclose(p32, pts, atol=1e-4 * max(1.0, np.abs(pts).max()))


def test_axis_aligned_plane_masks():
    box = np.array([47.0, 47.0, 37.2])
    for normal in ((0, 0, 1), (0, 1, 0), (1, 0, 0), (1, 1, 0)):
        for n in (1, 2, 64, 511, 512):
            g = R.plane_grid(box, (0, 0, 0), normal, n)
            _, mask = og.slice_points(box, (0, 0, 0), normal, n)
            np.testing.assert_array_equal(_device_mask(g), mask)


def test_volume_grid_record_positions():
    dims, origin, h = R.volume_grid(np.array([10.0, 12.0, 7.0]), 16)
    d2, o2, h2 = og.volume_points(np.array([10.0, 12.0, 7.0]), maxdim=16)
    np.testing.assert_array_equal(dims, d2)
    np.testing.assert_allclose(origin, o2)
    assert h == h2
    g = R.volume_grid_record(origin, h, dims, 2, 5)
    nx, ny, nz = dims
    assert (g["n_i"], g["n_j"], g["n_k"]) == (ny, nz, 3)
    assert g["out_offset"] == 2 * ny * nz
    # sample (i=y, j=z, k) sits at (x[2+k], y[i], z[j])
    p = g["origin"] + 1 * g["step_k"] + 3 * g["step_i"] + 4 * g["step_j"]
    np.testing.assert_allclose(p, origin + h * np.array([3, 3, 4]), atol=1e-5)


def test_tile_planner_covers_every_sample():
    grids = np.zeros(3, dtype=N.GRID_DTYPE)
    grids["n_i"], grids["n_j"], grids["n_k"] = [100, 1, 33], [70, 5000, 40], [1, 1, 3]
    grids["flags"][1] = N.MR_GRID_POINTS
    tiles = N.plan_tiles(grids)
    ti, tj = N.tile_shape()
    cover = {0: set(), 2: set()}
    pts = set()
    for t in tiles:
        if t["grid"] == 1:
            pts.update(range(t["j0"], min(5000, t["j0"] + ti * tj // 4 * 4)))
            continue
        G_ = grids[t["grid"]]
        for i in range(t["i0"], min(G_["n_i"], t["i0"] + ti)):
            for j in range(t["j0"], min(G_["n_j"], t["j0"] + tj)):
                cover[t["grid"]].add((i, j, t["k"]))
    assert len(cover[0]) == 100 * 70 and len(cover[2]) == 33 * 40 * 3
    assert pts == set(range(5000))
    assert len(N.plan_tiles(np.zeros(0, dtype=N.GRID_DTYPE))) == 0


def test_filter_tables_mirror_the_rfft_half():
    H, n_fft = R.ramp_response(486, 1.0, "shepp-logan")
    half = H[: n_fft // 2 + 1]
    full = np.concatenate([half, half[1:n_fft - n_fft // 2][::-1]])
    assert len(full) == n_fft == 1024
    np.testing.assert_array_equal(full[: n_fft // 2 + 1], half)
    np.testing.assert_array_equal(full[n_fft - np.arange(1, n_fft // 2)], half[1:n_fft // 2])


def test_stream_arrival_order_matches_reference():
    g = golden("misc.npz")
    for n in (1, 2, 10, 17, 64, 600):
        np.testing.assert_array_equal(S.arrival_order(n, "interleaved"), g[f"order_{n}"])
    np.testing.assert_array_equal(S.arrival_order(5), np.arange(5))
    with pytest.raises(ValueError):
        S.arrival_order(5, "random")


def test_cross3_is_numpy_cross_bit_for_bit():
    rng = np.random.default_rng(3)
    for _ in range(20000):
        a = rng.normal(size=3) * 10.0 ** rng.uniform(-4, 4)
        b = rng.normal(size=3) * 10.0 ** rng.uniform(-4, 4)
        assert np.cross(a, b).tobytes() == R._cross3(a, b).tobytes()
    for normal in ((0, 0, 1), (0, 1, 0), (1, 0, 0), (1, 1, 0), (0.3, -0.2, 0.9)):
        n = np.asarray(normal, float) / np.linalg.norm(normal)
        z = np.array([0.0, 0.0, 1.0])
        e1 = np.cross(z, n) if abs(n @ z) < 0.9 else np.cross(n, np.array([0.0, 1.0, 0.0]))
        e1 /= np.linalg.norm(e1)
        for x, y in zip(R.plane_basis(normal), (n, e1, np.cross(n, e1))):
            assert x.tobytes() == y.tobytes()


def test_orbit_filter_records_equal_per_call_records():
    """The reconstructor computes the filter records of the whole orbit once and copies
    rows per call; they must be the bytes a per-call computation gives."""
    K = R.cone_constants(G.circular_cone_vectors(120, 440.0, 680.0, 48, 60, 0.3).vectors)
    full = R.cone_filter_views(K, 48, 60, 128, 0)
    rng = np.random.default_rng(5)
    for t in range(40):
        k = int(rng.integers(1, 120))
        if t % 2:
            idx = np.sort(rng.choice(120, k, replace=False))
        else:
            a = int(rng.integers(0, 120 - k + 1))
            idx = np.arange(a, a + k)
        slots = np.arange(7, 7 + k)
        want = R.cone_filter_views({key: val[idx] for key, val in K.items()}, 48, 60, 128, slots)
        got = full[idx]
        got["slot"] = slots
        assert got.tobytes() == want.tobytes()


def test_first_of_run():
    f = R.SliceReconstructor._first_of_run
    assert f(np.arange(5, 9)) == 5
    assert f(np.array([3])) == 3
    assert f(np.array([3, 4])) == 3
    assert f(np.array([4, 3])) is None
    assert f(np.array([0, 2, 1, 3])) is None          # right span, wrong order
    assert f(np.array([0, 1, 3])) is None


def test_band_ordered_tiles_are_a_permutation_sorted_by_height():
    rng = np.random.default_rng(9)
    box = np.array([47.0, 47.0, 37.2])
    grids = np.zeros(3, dtype=N.GRID_DTYPE)
    for r in range(3):
        nrm = rng.normal(size=3)
        grids[r] = R.plane_grid(box, rng.uniform(-10, 10, 3), nrm / np.linalg.norm(nrm), 200)
    plain = N.plan_tiles(grids)
    axis = (0.0, 0.0, 1.0)
    banded = N.plan_tiles(grids, axis)
    assert sorted(map(bytes, plain)) == sorted(map(bytes, banded))
    ti, tj = N.tile_shape()
    g = grids[banded["grid"]]
    centre = (g["origin"].astype(np.float64) + (banded["i0"] + (ti - 1) / 2)[:, None] * g["step_i"]
              + (banded["j0"] + (tj - 1) / 2)[:, None] * g["step_j"])
    assert np.all(np.diff(centre[:, 2]) <= 1e-9)          # highest first, across the grids
    assert len(set(banded["grid"][:20])) > 1              # the grids are interleaved
    # point lists keep the planner's order
    pts = grids.copy()
    pts["flags"][1] = N.MR_GRID_POINTS
    assert N.plan_tiles(pts, axis).tobytes() == N.plan_tiles(pts).tobytes()


def test_product_phantom_matches_reference():
    """The torch chord-length projectors of the product phantom reproduce the reference's
    own phantom outputs (densities, line integrals, parallel and cone projections)."""
    import torch
    from tomography_local_demo_b200 import phantom as PH
    g = golden("phantom.npz")
    ph = PH.EllipsoidPhantom(scale=50.0)
    np.testing.assert_allclose(ph.evaluate(g["pts"]), g["evaluate"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(ph.line_integrals(g["starts"], g["dirs"]), g["lines"], rtol=1e-12, atol=1e-12)
    pg = G.ParallelGeometry(np.arange(9) * np.pi / 9, 10, 12, 9.0, 11.0)
    par = PH.project_parallel_torch(ph, pg).numpy()
    assert par.shape == g["par"].shape and par.dtype == np.float32
    np.testing.assert_allclose(par, g["par"], rtol=1e-6, atol=1e-6 * np.abs(g["par"]).max())
    cg = G.circular_cone_vectors(9, 300.0, 600.0, 10, 12, 15.0, det_shift_u=1.5)
    cone = PH.project_cone_torch(ph, cg, device="cpu").permute(1, 0, 2).numpy()
    np.testing.assert_allclose(cone, g["cone"], rtol=1e-6, atol=1e-6 * np.abs(g["cone"]).max())
    assert torch.get_default_dtype() == torch.float32


def test_acquisition_schedule_and_feeder():
    """Groups in arrival order, group k due when the views before it are (rate views/s),
    all at once for rate <= 0; the Feeder pushes every view once, in that order, and a
    stop() ends it before the next group."""
    sc = S.AcquisitionSchedule(10, "interleaved", group=4, rate=8.0)
    assert [len(g) for g in sc.groups] == [4, 4, 2]
    np.testing.assert_array_equal(np.concatenate(sc.groups), S.arrival_order(10, "interleaved"))
    np.testing.assert_allclose(sc.due, [0.0, 0.5, 1.0])
    assert [sc.due_by(t) for t in (0.0, 0.49, 0.5, 0.99, 5.0)] == [1, 1, 2, 2, 3]
    assert (S.AcquisitionSchedule(5, group=2, rate=0).due == 0).all()
    assert list(S.arrival_order(1, "interleaved")) == [0] and len(S.arrival_order(0, "interleaved")) == 0

    class Sink:
        def __init__(self):
            self.calls = []

        def add_projections(self, idx, block):
            self.calls.append((np.array(idx), np.array(block)))

    proj = np.arange(3 * 7 * 2, dtype=np.float32).reshape(3, 7, 2)
    sink = Sink()
    f = S.Feeder(sink, proj, order="interleaved", group=3, rate=0, verbose=False)
    f.run()
    assert f.sent == 7 and [len(i) for i, _ in sink.calls] == [3, 3, 1]
    for idx, blk in sink.calls:
        np.testing.assert_array_equal(blk, proj[:, idx, :])
    slow = Sink()
    f = S.Feeder(slow, proj, group=1, rate=2.0, verbose=False)
    f.start()
    f.stop()
    f.join(5)
    assert not f.is_alive() and f.stopped and len(slow.calls) <= 1


def test_ring_pitch_rows_start_32_byte_aligned():
    """The ring's row pitch is the smallest multiple of 32 bytes holding the row, for every
    store type (the tensor-core filter stores each row in 32-byte pieces)."""
    for cols in (1, 7, 8, 15, 16, 17, 486, 488, 496, 512, 1944):
        for store, esz in (("fp32", 4), ("bf16", 2), ("fp16", 2)):
            p = R.ring_pitch(cols, store)
            assert p >= cols and (p * esz) % 32 == 0
            assert p - 32 // esz < cols                   # the smallest such multiple
    assert R.ring_pitch(486, "bf16") == 496 and R.ring_pitch(486, "fp32") == 488
