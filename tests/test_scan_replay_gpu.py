"""SliceReconstructor.scan_replay: the ingest + batched back-projection of a resident scan,
captured once as a CUDA graph and replayed. A replay must give bit for bit what the eager
calls give (reset, add_raw_projections of the whole device buffer, reconstruct_planes_
tensor), follow new counts written into the same buffer, and leave the reconstructor
holding the scan for further requests."""
import numpy as np
import pytest
import torch

from tomography_local_demo_b200 import SliceReconstructor, circular_cone_vectors

pytestmark = pytest.mark.gpu

REQS = [dict(origin=(0.5, -1.0, 0.3), normal=(0.2, 0.3, 1.0), n=40),
        dict(origin=(0.0, 0.0, 0.0), normal=(1.0, 0.0, 0.0), n=32, zoom=2.0, cor_shift=0.7)]


def _scan(seed, k=48, rows=24, cols=36):
    rng = np.random.default_rng(seed)
    raw = rng.integers(2000, 45000, (k, rows, cols)).astype(np.uint16)
    return torch.from_numpy(raw.view(np.int16)).cuda()


@pytest.mark.parametrize("store,filt", [("bf16", "tc"), ("fp32", "fft"), ("fp16", "tc")])
def test_replay_equals_the_eager_calls(cuda, store, filt):
    geom = circular_cone_vectors(48, 300.0, 600.0, 24, 36, 3.0)
    rng = np.random.default_rng(3)
    flat = rng.normal(50000, 500, (2, 24, 36)).clip(0, 65535).astype(np.uint16)
    dark = rng.normal(100, 5, (2, 24, 36)).clip(0, 65535).astype(np.uint16)

    def eager(raw):
        rec = SliceReconstructor(None, geom, verbose=False, store=store, filter=filt)
        rec.set_flat_dark(flat, dark)
        rec.add_raw_projections(np.arange(raw.shape[0]), raw)
        return [t.clone() for t in rec.reconstruct_planes_tensor(REQS)]

    buf = _scan(11)
    rec = SliceReconstructor(None, geom, verbose=False, store=store, filter=filt)
    rec.set_flat_dark(flat, dark)
    rep = rec.scan_replay(buf, REQS)
    for seed in (11, 12):
        buf.copy_(_scan(seed))                      # the next scan lands in the same buffer
        got = [t.clone() for t in rep.replay()]
        torch.cuda.synchronize()
        want = eager(buf)
        for g, w in zip(got, want):
            assert torch.count_nonzero(w) > 0
            assert torch.equal(g, w)
        assert rec.n == 48
        # the reconstructor serves further requests from the replayed scan
        other = [dict(origin=(1.0, 0.0, 0.0), normal=(0.0, 1.0, 1.0), n=24)]
        ref = SliceReconstructor(None, geom, verbose=False, store=store, filter=filt)
        ref.set_flat_dark(flat, dark)
        ref.add_raw_projections(np.arange(48), buf)
        assert torch.equal(rec.reconstruct_planes_tensor(other)[0], ref.reconstruct_planes_tensor(other)[0])
    # another scan order through the eager calls, then a replay: the replay restores its
    # own view records
    rec.reset()
    order = np.arange(48)[::-1].copy()
    rec.add_raw_projections(order, buf[torch.from_numpy(order).cuda()])
    got = [t.clone() for t in rep.replay()]
    for g, w in zip(got, eager(buf)):
        assert torch.equal(g, w)


def test_replay_arguments(cuda):
    geom = circular_cone_vectors(8, 300.0, 600.0, 8, 8, 3.0)
    rec = SliceReconstructor(None, geom, verbose=False)
    raw = torch.zeros((8, 8, 8), dtype=torch.int16, device="cuda")
    with pytest.raises(RuntimeError):
        rec.scan_replay(raw, REQS)                  # no flat / dark yet
    rec.set_flat_dark(np.full((8, 8), 50000, np.uint16), np.full((8, 8), 100, np.uint16))
    with pytest.raises(ValueError):
        rec.scan_replay(raw.cpu(), REQS)
    with pytest.raises(ValueError):
        rec.scan_replay(torch.zeros((9, 8, 8), dtype=torch.int16, device="cuda"), REQS)
    with pytest.raises(ValueError):
        rec.scan_replay(raw.float(), REQS)
    rep = rec.scan_replay(raw, REQS)
    rec.set_flat_dark(np.full((8, 8), 40000, np.uint16), np.full((8, 8), 100, np.uint16))
    with pytest.raises(RuntimeError):
        rep.replay()
