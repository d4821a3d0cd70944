"""Continuously batched slice server: every result equals the same request reconstructed
alone (bit for bit - the per-tile arithmetic and the cluster reduction order do not
depend on the batch), memory-based admission, and serving while projections stream in."""
import threading

import numpy as np
import pytest

from oracle import phantom as oph
from tomography_local_demo_b200 import SliceReconstructor, circular_cone_vectors
from tomography_local_demo_b200.server import SliceServer
from tomography_local_demo_b200.stream import arrival_order

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scan():
    geom = circular_cone_vectors(96, 300.0, 600.0, 64, 80, 3.0)
    proj = oph.project_cone(oph.Phantom(scale=50.0), geom.vectors, 64, 80)
    return geom, proj


def random_requests(rng, k):
    reqs = []
    for _ in range(k):
        nrm = rng.normal(size=3)
        reqs.append(dict(origin=tuple(rng.uniform(-10, 10, 3)), normal=tuple(nrm),
                         n=int(rng.choice([32, 64, 128, 256])), zoom=float(rng.uniform(1, 8)),
                         cor_shift=float(rng.uniform(-10, 10))))
    return reqs


@pytest.mark.parametrize("store,graphs", [("fp32", True), ("bf16", True), ("bf16", False)])
def test_each_result_is_the_same_alone_and_in_the_mix(cuda, scan, store, graphs):
    geom, proj = scan
    rec = SliceReconstructor(proj, geom, verbose=False, store=store)
    rng = np.random.default_rng(0)
    reqs = random_requests(rng, 40)
    srv = SliceServer(rec, budget_bytes=64 << 20, max_batch=16, use_graphs=graphs)
    try:
        futs = [srv.submit(**r) for r in reqs]
        prev = srv.submit_preview(24)
        mixed = [f.result(timeout=60) for f in futs]
        vol, origin, h = prev.result(timeout=60)
        srv.device_status()
    finally:
        srv.close()
    assert srv.batches >= 3                                  # the budget forced several batches
    for r, img in zip(reqs, mixed):
        alone = rec.reconstruct_planes_tensor([r])[0].cpu().numpy()
        np.testing.assert_array_equal(img, alone)
    want, _, _ = rec.reconstruct_volume(maxdim=24)
    np.testing.assert_allclose(vol, want, rtol=0, atol=1e-6 * np.abs(want).max())
    st = srv.stats()
    assert st["requests"] == len(reqs) + 1 and st["p99_ms"] >= st["p50_ms"] > 0


def test_admission_rejects_requests_over_budget(cuda, scan):
    geom, proj = scan
    rec = SliceReconstructor(proj, geom, verbose=False)
    srv = SliceServer(rec, budget_bytes=100_000, pool_bytes=1 << 20)
    try:
        big = srv.submit((0, 0, 0), (0, 0, 1), n=512)          # 1 MB > 100 kB budget
        with pytest.raises(MemoryError):
            big.result(timeout=10)
        small = [srv.submit((0, 0, z), (0, 0, 1), n=100) for z in (-3, 0, 3)]   # 40 kB each
        imgs = [f.result(timeout=30) for f in small]
    finally:
        srv.close()
    assert 2 <= srv.batches <= 3                             # at most two 40 kB slices fit 100 kB
    for z, img in zip((-3, 0, 3), imgs):
        np.testing.assert_array_equal(img, rec.reconstruct_planes_tensor(
            [dict(origin=(0, 0, z), normal=(0, 0, 1), n=100)])[0].cpu().numpy())


def test_serving_while_projections_stream_in(cuda, scan):
    geom, proj = scan
    rec = SliceReconstructor(None, geom, verbose=False, store="bf16")
    srv = SliceServer(rec, budget_bytes=32 << 20)
    order = arrival_order(geom.n_angles, "interleaved")
    rng = np.random.default_rng(1)
    seen = []
    try:
        def feed():
            for i in range(0, len(order), 8):
                rec.add_projections(order[i:i + 8], proj[:, order[i:i + 8], :])
        th = threading.Thread(target=feed)
        th.start()
        while th.is_alive():
            seen.append(srv.submit(**random_requests(rng, 1)[0]).result(timeout=30))
        th.join()
        final = srv.submit((0, 0, 0), (0.1, 0.2, 1.0), n=64).result(timeout=30)
    finally:
        srv.close()
    assert rec.n == geom.n_angles and len(seen) > 0
    want = rec.reconstruct_planes_tensor([dict(origin=(0, 0, 0), normal=(0.1, 0.2, 1.0), n=64)])[0].cpu().numpy()
    np.testing.assert_array_equal(final, want)
