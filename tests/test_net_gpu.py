"""The wire-compatible slice service end to end over 127.0.0.1: an adapter pushes float
and raw projections, viewers get the same slices (FP32 bit for bit, BF16 as the rounded
FP32 image), previews, COR changes and the reference's error replies."""
import threading

import numpy as np
import pytest
import torch

from oracle import phantom as oph
from tomography_local_demo_b200 import SliceReconstructor, circular_cone_vectors, net
from tomography_local_demo_b200.stream import arrival_order

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(600)]


@pytest.fixture()
def server(cuda):
    srv = net.Server(port=0, verbose=False, store="bf16", filter="tc", budget_bytes=1 << 30)
    address = srv.listen()
    t = threading.Thread(target=srv.serve_forever, daemon=True)
    t.start()
    yield srv, address
    srv.close()


REQS = [dict(origin=(1.0, -2.0, 0.5), normal=(0.3, 0.2, 1.0), n=48, zoom=1.5),
        dict(origin=(0.0, 0.0, 0.0), normal=(1.0, 0.0, 0.0), n=32, zoom=1.0),
        dict(origin=(-3.0, 1.0, 2.0), normal=(0.1, -0.7, 0.4), n=64, zoom=2.0)]


def _local(rec, r):
    return rec.reconstruct_planes_tensor([dict(r)])[0].cpu().numpy()


def test_float_projections_slices_previews_and_cor(server):
    srv, address = server
    geom = circular_cone_vectors(60, 300.0, 600.0, 32, 40, 2.0)
    proj = oph.project_cone(oph.Phantom(scale=40.0), geom.vectors, 32, 40).astype(np.float32)
    order = arrival_order(60, "interleaved")
    local = SliceReconstructor(None, geom, verbose=False, store="bf16", filter="tc")
    sink = net.RemoteSink(address, geom)
    for part in np.array_split(order, 4):
        assert sink.add_projections(part, proj[:, part, :]) == local.add_projections(part, proj[:, part, :])
    sink.end()

    view = net.RemoteReconstructor(address)
    assert view.n == 60 and view.kind == "cone" and view.n_total == 60
    np.testing.assert_array_equal(view.box, local.box)
    for r in REQS:
        img, pts = view.reconstruct_plane(r["origin"], r["normal"], n=r["n"], zoom=r["zoom"])
        want = _local(local, r)
        np.testing.assert_array_equal(img, want.astype(np.float64))
        assert pts.shape == (r["n"], r["n"], 3)
    batch = view.reconstruct_planes(REQS)
    for r, img in zip(REQS, batch):
        np.testing.assert_array_equal(img, _local(local, r).astype(np.float64))

    view16 = net.RemoteReconstructor(address, encoding="bf16")
    for r in REQS:
        img, _ = view16.reconstruct_plane(r["origin"], r["normal"], n=r["n"], zoom=r["zoom"])
        data, extra = net.encode_image(_local(local, r), "bf16")
        np.testing.assert_array_equal(img, net.decode_image(extra, data).astype(np.float64))

    vol, origin, h = view.preview_volume(24)
    want, worigin, wh = local.reconstruct_volume(maxdim=24)
    np.testing.assert_allclose(vol, want, rtol=0, atol=1e-6 * np.abs(want).max())
    np.testing.assert_allclose(origin, worigin)
    assert h == pytest.approx(wh)

    view.set_cor_shift(1.25)
    local.set_cor_shift(1.25)
    assert view.cor_shift == 1.25
    r = REQS[0]
    img, _ = view.reconstruct_plane(r["origin"], r["normal"], n=r["n"], zoom=r["zoom"])
    np.testing.assert_array_equal(img, _local(local, r).astype(np.float64))
    best, _ = view.estimate_cor(verbose=False)
    assert best == local.estimate_cor(verbose=False)[0]
    for c in (view, view16, sink):
        c.close()


def test_raw_projections_through_the_fused_ingest(server):
    srv, address = server
    geom = circular_cone_vectors(40, 300.0, 600.0, 24, 36, 3.0)
    rng = np.random.default_rng(4)
    raw = rng.integers(2000, 45000, (40, 48, 72)).astype(np.uint16)
    flat = rng.normal(50000, 500, (2, 48, 72)).clip(0, 65535).astype(np.uint16)
    dark = rng.normal(100, 5, (2, 48, 72)).clip(0, 65535).astype(np.uint16)
    local = SliceReconstructor(None, geom, verbose=False, store="bf16", filter="tc")
    local.set_flat_dark(flat, dark, bin=2, flip_rows=True)
    sink = net.RemoteSink(address, geom)
    sink.set_flat_dark(flat, dark, bin=2, flip_rows=True)
    order = arrival_order(40, "interleaved")
    for part in (order[:25], order[20:]):                   # 5 views sent twice (dedup)
        n_remote = sink.add_raw_projections(part, raw[part])
        assert n_remote == local.add_raw_projections(part, torch.from_numpy(raw[part].view(np.int16)).cuda())
    view = net.RemoteReconstructor(address)
    assert view.n == 40
    want = [_local(local, r).astype(np.float64) for r in REQS]
    for r, w in zip(REQS, want):
        img, _ = view.reconstruct_plane(r["origin"], r["normal"], n=r["n"], zoom=r["zoom"])
        np.testing.assert_array_equal(img, w)
    sink.reset()                                            # a new scan, same geometry
    assert view.n == 0
    sink.add_raw_projections(order, raw[order])
    for got, w in zip(view.reconstruct_planes(REQS), want):
        np.testing.assert_array_equal(got, w)
    view.close()
    sink.close()


def test_errors_come_back_as_the_reference_replies(server):
    srv, address = server
    c = net._Conn(address, "viewer")
    h, _ = c.call({"cmd": "info"})
    assert h == {"ready": False}
    with pytest.raises(RuntimeError, match="no scan yet"):
        c.call({"cmd": "slice", "origin": [0, 0, 0], "normal": [0, 0, 1], "n": 16})
    c2 = net._Conn(address, "viewer")                   # the failed connection was closed
    with pytest.raises(RuntimeError, match="unknown command"):
        c2.call({"cmd": "no-such-command"})
    c.close()
    c2.close()
