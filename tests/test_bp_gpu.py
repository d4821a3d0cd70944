"""Back-projection kernel (mr_backproject) against the C oracle of minirecast's Numba
kernels, on seeded inputs (noise-like stacks, the hardest case for FP32 coordinates).
Tolerances: rel-L2 <= 5e-5 against the oracle on the same stack (the product bar is
1e-4 against the reference); BF16/FP16 stores are checked against the oracle fed the
same rounded stack (5e-5) and against the FP32 stack (stated bounds)."""
import numpy as np
import pytest

from conftest import rel_l2
from gpu_helpers import DeviceRing
from oracle import bp as obp
from oracle import filter as of
from oracle import geometry as og
from tomography_local_demo_b200 import _native as N
from tomography_local_demo_b200 import recon as R

pytestmark = pytest.mark.gpu


def cone_case(A=48, rows=40, cols=56, seed=0, jitter=0.02):
    rng = np.random.default_rng(seed)
    V = og.circular_cone_vectors(A, 120.0, 200.0, 1.0, det_shift_u=0.6)
    V = V + rng.normal(0.0, jitter, V.shape)
    # smooth-ish stack: low-pass noise, like filtered projections of a phantom
    q = rng.normal(0.0, 1.0, (A, rows, cols))
    q = (q + np.roll(q, 1, 2) + np.roll(q, 1, 1)).astype(np.float32)
    return V, q, rows, cols


def oracle_cone(V, q, pts, n_views, shift=0.0):
    K = of.cone_constants(V[:n_views])
    D = K["d"] - shift * K["u"] if shift else K["d"]
    return obp.bp_cone(q[:n_views], K["s"], D, K["uu"], K["vv"], K["n"], K["sdd"], K["sod"], pts,
                       np.pi / n_views)


@pytest.mark.parametrize("shift", [0.0, 2.3])
def test_cone_points_match_oracle(cuda, shift):
    V, q, rows, cols = cone_case()
    ring = DeviceRing(q, R.cone_view_maps(R.cone_constants(V), rows, cols), N.MR_CONE)
    rng = np.random.default_rng(1)
    pts = rng.uniform(-22, 22, (5000, 3))
    got = ring.points(pts, len(V), np.pi / len(V), shift)
    want = oracle_cone(V, q, pts, len(V), shift)
    assert rel_l2(got, want) < 5e-5
    assert np.max(np.abs(got - want)) < 1e-4 * np.max(np.abs(want))


def test_cone_snapshot_uses_first_n_views(cuda):
    V, q, rows, cols = cone_case(seed=4)
    ring = DeviceRing(q, R.cone_view_maps(R.cone_constants(V), rows, cols), N.MR_CONE)
    pts = np.random.default_rng(2).uniform(-20, 20, (777, 3))
    for n in (1, 7, 31):
        got = ring.points(pts, n, np.pi / n)
        assert rel_l2(got, oracle_cone(V, q, pts, n)) < 5e-5
    assert np.all(ring.points(pts, 0, 0.0) == 0.0)


@pytest.mark.parametrize("kernel", ["staged", "plain"])
@pytest.mark.parametrize("seed", range(4))
def test_cone_planes_match_oracle_with_exact_mask(cuda, seed, kernel):
    V, q, rows, cols = cone_case(seed=seed)
    box = og.cone_volume_box(V, rows, cols)
    ring = DeviceRing(q, R.cone_view_maps(R.cone_constants(V), rows, cols), N.MR_CONE)
    rng = np.random.default_rng(10 + seed)
    reqs = []
    for r in range(5):                 # several grids of different sizes in ONE launch
        reqs.append(dict(origin=rng.uniform(-5, 5, 3), normal=rng.normal(size=3),
                         n=int(rng.integers(5, 90)), zoom=float(rng.uniform(0.3, 8.0)),
                         center=None if r % 2 else rng.uniform(-3, 3, 3),
                         cor_shift=float(rng.uniform(-3, 3))))
    grids = np.zeros(len(reqs), N.GRID_DTYPE)
    off = 0
    for r, rq in enumerate(reqs):
        grids[r] = R.plane_grid(box, rq["origin"], rq["normal"], rq["n"], None, rq["zoom"],
                                rq["center"], rq["cor_shift"])
        grids[r]["out_offset"] = off
        off += rq["n"] ** 2
    grids["n_views"] = len(V)
    grids["scale"] = np.pi / len(V)
    out = ring.run(grids, off, kernel)
    off = 0
    for rq in reqs:
        n = rq["n"]
        img = out[off:off + n * n].reshape(n, n)
        off += n * n
        pts, mask = og.slice_points(box, rq["origin"], rq["normal"], n, None, rq["zoom"], rq["center"])
        want = np.zeros(n * n)
        if mask.any():
            want[mask.ravel()] = oracle_cone(V, q, pts.reshape(-1, 3)[mask.ravel()], len(V), rq["cor_shift"])
        want = want.reshape(n, n)
        assert np.all(img[~mask] == 0.0)
        if mask.any():
            assert rel_l2(img[mask], want[mask]) < 5e-5


@pytest.mark.parametrize("kernel", ["staged", "plain"])
def test_cone_volume_grid_matches_oracle(cuda, kernel):
    V, q, rows, cols = cone_case(A=30, seed=7)
    box = og.cone_volume_box(V, rows, cols)
    ring = DeviceRing(q, R.cone_view_maps(R.cone_constants(V), rows, cols), N.MR_CONE)
    dims, origin, h = R.volume_grid(box, 37)
    nx, ny, nz = dims
    grids = np.zeros(2, N.GRID_DTYPE)
    grids[0] = R.volume_grid_record(origin, h, dims, 0, 11)      # two x-slabs, one launch
    grids[1] = R.volume_grid_record(origin, h, dims, 11, nx)
    grids["n_views"], grids["scale"] = len(V), np.pi / len(V)
    vol = ring.run(grids, nx * ny * nz, kernel).reshape(nx, ny, nz)
    x, y, z = (origin[i] + h * np.arange(dims[i]) for i in range(3))
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    want = oracle_cone(V, q, np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1), len(V)).reshape(nx, ny, nz)
    assert rel_l2(vol, want) < 5e-5


@pytest.mark.parametrize("kernel", ["staged", "plain"])
@pytest.mark.parametrize("shift", [0.0, -1.3])
def test_parallel_points_and_planes_match_oracle(cuda, shift, kernel):
    rng = np.random.default_rng(5)
    A, rows, cols = 60, 30, 44
    ang = np.arange(A) * np.pi / A
    q = rng.normal(0, 1, (A, rows, cols)).astype(np.float32)
    ring = DeviceRing(q, R.parallel_view_maps(ang, 0.9, 1.1, rows, cols), N.MR_PARALLEL)
    pts = rng.uniform(-20, 20, (3000, 3))
    got = ring.points(pts, A, np.pi / A, shift)
    want = obp.bp_parallel(q, np.cos(ang), np.sin(ang), 0.9, 1.1, pts, np.pi / A, shift)
    assert rel_l2(got, want) < 5e-5
    box = og.parallel_volume_box(rows, cols, 0.9, 1.1)
    g = np.zeros(1, N.GRID_DTYPE)
    g[0] = R.plane_grid(box, (1, 2, 3), (0.2, 1.0, 0.4), 50, None, 1.3, None, shift)
    g["n_views"], g["scale"] = A, np.pi / A
    img = ring.run(g, 2500, kernel).reshape(50, 50)
    pts, mask = og.slice_points(box, (1, 2, 3), (0.2, 1.0, 0.4), 50, None, 1.3, None)
    want = obp.bp_parallel(q, np.cos(ang), np.sin(ang), 0.9, 1.1, pts.reshape(-1, 3), np.pi / A,
                           shift).reshape(50, 50)
    assert np.all(img[~mask] == 0)
    assert rel_l2(img[mask], want[mask]) < 5e-5


@pytest.mark.parametrize("store,bound", [("bf16", 5e-3), ("fp16", 1e-3)])
def test_low_precision_stores(cuda, store, bound):
    V, q, rows, cols = cone_case(seed=9)
    maps = R.cone_view_maps(R.cone_constants(V), rows, cols)
    ring = DeviceRing(q, maps, N.MR_CONE, store=store)
    pts = np.random.default_rng(3).uniform(-20, 20, (4000, 3))
    got = ring.points(pts, len(V), np.pi / len(V))
    # kernel arithmetic: exact against the oracle fed the same rounded stack
    assert rel_l2(got, oracle_cone(V, ring.stored.astype(np.float32), pts, len(V))) < 5e-5
    # storage error against the FP32 stack (white-noise stack: the worst case)
    assert rel_l2(got, oracle_cone(V, q, pts, len(V))) < bound


def test_fp16_per_view_scale(cuda):
    V, q, rows, cols = cone_case(seed=11)
    q = q * np.linspace(1e3, 3e4, len(V))[:, None, None].astype(np.float32)   # beyond fp16 range
    qs = 2.0 ** np.ceil(np.log2(np.abs(q).max(axis=(1, 2)) / 16384.0))
    ring = DeviceRing(q, R.cone_view_maps(R.cone_constants(V), rows, cols), N.MR_CONE, "fp16", qs)
    pts = np.random.default_rng(3).uniform(-20, 20, (2000, 3))
    got = ring.points(pts, len(V), np.pi / len(V))
    assert rel_l2(got, oracle_cone(V, q, pts, len(V))) < 1e-3


def test_points_far_outside_detector_are_zero(cuda):
    V, q, rows, cols = cone_case(seed=2)
    ring = DeviceRing(q, R.cone_view_maps(R.cone_constants(V), rows, cols), N.MR_CONE)
    pts = np.array([[500.0, 0, 0], [0, 0, 300.0], [0, 0, -300.0], [1e4, 1e4, 1e4]])
    got = ring.points(pts, len(V), 1.0)
    want = oracle_cone(V, q, pts, len(V)) * len(V) / np.pi
    np.testing.assert_allclose(got, want, atol=1e-5 * max(1.0, np.abs(want).max()))


@pytest.mark.parametrize("store", ["fp32", "bf16", "fp16"])
def test_staged_kernel_edge_footprints(cuda, store):
    """Planes whose tile footprints are larger than a stage (zoomed out: global-load
    fallback), partly or wholly off the detector (TMA zero fill / skipped views), tiny
    (zoom 8) and grids larger than the box: staged == plain == oracle on the stored stack."""
    A, rows, cols = 40, 48, 64
    rng = np.random.default_rng(21)
    V = og.circular_cone_vectors(A, 150.0, 250.0, 1.0) + rng.normal(0, 0.01, (A, 12))
    q = rng.normal(0, 1, (A, rows, cols)).astype(np.float32)
    ring = DeviceRing(q, R.cone_view_maps(R.cone_constants(V), rows, cols), N.MR_CONE, store)
    box = og.cone_volume_box(V, rows, cols) * np.array([1.6, 1.6, 1.8])   # larger than the FOV
    cases = [((0, 0, 0), (0, 0, 1), 96, 0.25), ((5, 3, -2), (0.3, 1.0, 0.2), 70, 1.0),
             ((0, 0, 30), (1, 0, 0.1), 64, 0.6), ((2, 2, 2), (0.5, 0.5, 0.7), 128, 8.0),
             ((0, 0, 0), (0.01, 0.02, 1.0), 33, 2.5)]
    grids = np.zeros(len(cases), N.GRID_DTYPE)
    off = 0
    for r, (o, nrm, n, zm) in enumerate(cases):
        grids[r] = R.plane_grid(box, o, nrm, n, None, zm, None, 0.0)
        grids[r]["out_offset"] = off
        off += n * n
    grids["n_views"], grids["scale"] = A, np.pi / A
    staged = ring.run(grids, off, "staged")
    plain = ring.run(grids, off, "plain")
    assert rel_l2(staged, plain) < 5e-5
    off = 0
    stack = ring.stored.astype(np.float32)
    for o, nrm, n, zm in cases:
        pts, mask = og.slice_points(box, o, nrm, n, None, zm, None)
        img = staged[off:off + n * n].reshape(n, n)
        off += n * n
        want = oracle_cone(V, stack, pts.reshape(-1, 3)[mask.ravel()], A)
        assert np.all(img[~mask] == 0)
        assert rel_l2(img[mask], want) < 5e-5


@pytest.mark.parametrize("kernel", ["staged", "plain", "points"])
def test_view_ranges_accumulate_to_the_full_sum(cuda, kernel):
    """mr_grid.view_begin / accumulate: a sub-range of slots alone matches the oracle on
    those views, and ranges summed in order (the first writes, the rest add) equal the
    one-launch sum over all views to FP32 rounding, with the same zeros outside the box."""
    import torch
    V, q, rows, cols = cone_case(A=45, seed=13)
    box = og.cone_volume_box(V, rows, cols)
    ring = DeviceRing(q, R.cone_view_maps(R.cone_constants(V), rows, cols), N.MR_CONE)
    scale = np.pi / len(V)
    if kernel == "points":
        pts = np.random.default_rng(6).uniform(-20, 20, (3001, 3))
        p_dev = torch.from_numpy(pts.astype(np.float32)).to(ring.dev)
        g = np.zeros(1, N.GRID_DTYPE)
        g["n_i"], g["n_j"], g["n_k"] = 1, len(pts), 1
        g["flags"] = N.MR_GRID_POINTS
        g["out_stride_j"] = 1
        g["points"] = p_dev.data_ptr()
        n_out, kern = len(pts), "plain"
        mask = np.ones(len(pts), bool)
    else:
        g = np.zeros(2, N.GRID_DTYPE)
        g[0] = R.plane_grid(box, (1, -2, 0.5), (0.3, 0.2, 1.0), 61, None, 1.0, None, 0.4)
        g[1] = R.plane_grid(box, (0, 3, 1), (1.0, 0.1, 0.2), 47, None, 0.7, None, 0.0)
        g[1]["out_offset"] = 61 * 61
        n_out, kern = 61 * 61 + 47 * 47, kernel
        pts0, m0 = og.slice_points(box, (1, -2, 0.5), (0.3, 0.2, 1.0), 61, None, 1.0, None)
        mask = np.concatenate([m0.ravel(), og.slice_points(box, (0, 3, 1), (1.0, 0.1, 0.2), 47, None,
                                                           0.7, None)[1].ravel()])
    g["scale"] = scale
    full = g.copy()
    full["n_views"] = len(V)
    want = ring.run(full, n_out, kern)
    # one sub-range alone, against the oracle on those views
    sub = g.copy()
    sub["view_begin"], sub["n_views"] = 11, 17
    got_sub = ring.run(sub, n_out, kern)
    if kernel == "points":
        K = of.cone_constants(V[11:28])
        ref = obp.bp_cone(q[11:28], K["s"], K["d"], K["uu"], K["vv"], K["n"], K["sdd"], K["sod"],
                          pts, scale)
        assert rel_l2(got_sub, ref) < 5e-5
    else:
        ref = np.zeros(n_out)
        K = of.cone_constants(V[11:28])
        pts1 = og.slice_points(box, (0, 3, 1), (1.0, 0.1, 0.2), 47, None, 0.7, None)[0]
        D0 = K["d"] - 0.4 * K["u"]
        P0 = pts0.reshape(-1, 3)[m0.ravel()]
        ref[:61 * 61][m0.ravel()] = obp.bp_cone(q[11:28], K["s"], D0, K["uu"], K["vv"], K["n"], K["sdd"],
                                                K["sod"], P0, scale)
        m1 = mask[61 * 61:]
        ref[61 * 61:][m1] = obp.bp_cone(q[11:28], K["s"], K["d"], K["uu"], K["vv"], K["n"], K["sdd"],
                                        K["sod"], pts1.reshape(-1, 3)[m1], scale)
        assert np.all(got_sub[~mask] == 0)
        assert rel_l2(got_sub[mask], ref[mask]) < 5e-5
    # a range running past the ring is clamped to its slots: [40, 140) sums slots 40..44
    over = g.copy()
    over["view_begin"], over["n_views"] = 40, 100
    tail = g.copy()
    tail["view_begin"], tail["n_views"] = 40, 5
    np.testing.assert_array_equal(ring.run(over, n_out, kern), ring.run(tail, n_out, kern))
    # ranges summed in order into one buffer
    out = torch.full((n_out,), float("nan"), dtype=torch.float32, device=ring.dev)
    status = torch.zeros(1, dtype=torch.int32, device=ring.dev)
    st = torch.cuda.current_stream()
    for i, (a, b) in enumerate([(0, 7), (7, 30), (30, 31), (31, 45)]):
        part = g.copy()
        part["view_begin"], part["n_views"], part["accumulate"] = a, b - a, int(i > 0)
        R.backproject_device(ring.c, ring.views, part, out, st, ring.dev, kernel=kern, status=status)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    got = out.cpu().numpy().astype(np.float64)
    assert np.all(got[~mask] == 0) and np.all(want[~mask] == 0)
    assert rel_l2(got[mask], want[mask]) < 1e-6
