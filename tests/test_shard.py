"""Multi-GPU sharding (tomography_local_demo_b200.shard): the host logic with two gloo ranks
on CPU (spawned processes, rendezvous on 127.0.0.1) and a stand-in reconstructor whose
output is a known function of the plane / request index; on the GPU, the slab
reconstruction that each rank runs against the full volume."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from tomography_local_demo_b200 import shard


class FakeRec:
    """Volume of dims (7, 3, 2) whose plane k holds k + 0.5; slice requests of size n whose
    image holds n + 0.25 - the reconstruction calls the shard helpers make."""

    device = torch.device("cpu")

    def _volume_frame(self, voxel, maxdim):
        return (7, 3, 2), np.zeros(3), 1.0

    def reconstruct_volume_slab_tensor(self, k0, k1, voxel=None, maxdim=None):
        ks = torch.arange(k0, k1, dtype=torch.float32) + 0.5
        return ks[:, None, None].expand(k1 - k0, 3, 2).contiguous(), np.zeros(3), 1.0

    def reconstruct_planes_tensor(self, reqs):
        return [torch.full((r["n"], r["n"]), r["n"] + 0.25) for r in reqs]


def _worker(rank, world, port, out_dir):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        rec = FakeRec()
        vol, _, _ = shard.gather_volume(rec)
        reqs = [dict(n=n) for n in (4, 3, 5, 2, 6)]
        imgs = shard.gather_planes(rec, reqs)
        raw = torch.arange(12, dtype=torch.int16).reshape(3, 4) * (7 if rank == 0 else 0)
        shard.broadcast_views(raw)
        if rank == 0:
            np.save(os.path.join(out_dir, "vol.npy"), vol.numpy())
            np.save(os.path.join(out_dir, "imgs.npy"), np.array([float(im.mean()) for im in imgs]))
            np.save(os.path.join(out_dir, "shapes.npy"), np.array([im.shape[0] for im in imgs]))
        else:
            assert vol is None and imgs is None
        np.save(os.path.join(out_dir, f"raw{rank}.npy"), raw.numpy())
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_slab_bounds_partition_the_planes():
    for n in (1, 7, 8, 640):
        for world in (1, 2, 3, 8):
            spans = [shard.slab_bounds(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1


def test_shard_requests_round_robin():
    reqs = list(range(7))
    got = sorted(i for w in range(3) for i, _ in shard.shard_requests(reqs, w, 3))
    assert got == reqs
    assert [i for i, _ in shard.shard_requests(reqs, 1, 3)] == [1, 4]


def test_two_gloo_ranks_gather_volume_slices_and_broadcast_views(tmp_path):
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    vol = np.load(tmp_path / "vol.npy")
    assert vol.shape == (7, 3, 2)
    np.testing.assert_array_equal(vol[:, 0, 0], np.arange(7) + 0.5)
    np.testing.assert_array_equal(np.load(tmp_path / "shapes.npy"), [4, 3, 5, 2, 6])
    np.testing.assert_array_equal(np.load(tmp_path / "imgs.npy"), np.array([4, 3, 5, 2, 6]) + 0.25)
    want = np.arange(12).reshape(3, 4) * 7
    for r in (0, 1):
        np.testing.assert_array_equal(np.load(tmp_path / f"raw{r}.npy"), want)


@pytest.mark.gpu
def test_slabs_reproduce_the_full_volume(cuda):
    from oracle import phantom as oph
    from tomography_local_demo_b200 import SliceReconstructor, circular_cone_vectors
    geom = circular_cone_vectors(48, 300.0, 600.0, 32, 40, 3.0)
    proj = oph.project_cone(oph.Phantom(scale=40.0), geom.vectors, 32, 40)
    rec = SliceReconstructor(proj, geom, verbose=False)
    full, origin, h = rec.reconstruct_volume_tensor(maxdim=24)
    nx = full.shape[0]
    parts = [rec.reconstruct_volume_slab_tensor(*shard.slab_bounds(nx, r, 3), maxdim=24)[0] for r in range(3)]
    got = torch.cat(parts).cpu().numpy()
    want = full.cpu().numpy()
    assert got.shape == want.shape
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-5 * np.abs(want).max())
    vol, _, _ = shard.gather_volume(rec, maxdim=24)                   # single process: the slab is the volume
    np.testing.assert_array_equal(vol.cpu().numpy(), want)
