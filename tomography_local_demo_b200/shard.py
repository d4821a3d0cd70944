"""Multi-GPU sharding of the reconstruction path: one process per GPU (torch.distributed,
NCCL between GPUs; the same code runs over gloo on CPU tensors).

The work is independent per output voxel and per request (minirecast reconstructs each
slice and each z-slab on its own, recon.py:405-470), so it shards without any collective
on the data path: every rank holds a replica of the filtered-view ring and computes its
share of the requests or of the volume's x-planes. Collectives appear only at the two real
exchange steps:
  * broadcast_views: raw counts read by one rank (the acquisition host) reach every
    rank's ingest (NCCL broadcast over NVLink);
  * gather_* : results assembled on one rank (a full volume for the mesh export of
    model.py, a batch of slices for a viewer).
"""
import numpy as np
import torch
import torch.distributed as dist


def _rank_world(group):
    if not dist.is_available() or not dist.is_initialized():
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def slab_bounds(n, rank, world):
    """Planes [k0, k1) of rank `rank` when n planes are split into `world` contiguous
    slabs whose sizes differ by at most one."""
    base, extra = divmod(int(n), int(world))
    k0 = rank * base + min(rank, extra)
    return k0, k0 + base + (1 if rank < extra else 0)


def shard_requests(requests, rank, world):
    """(original index, request) pairs of this rank: round robin over the request list."""
    return [(i, r) for i, r in enumerate(requests) if i % world == rank]


def broadcast_views(raw, group=None, src=0):
    """Broadcast a tensor of raw counts (or any ingest block) from rank `src` in place;
    every rank passes a tensor of the same shape and dtype (on its own GPU for NCCL)."""
    if _rank_world(group)[1] > 1:
        if not raw.is_contiguous():
            raise ValueError("broadcast_views needs a contiguous tensor")
        # 16-bit counts travel as bytes: neither NCCL nor gloo has a 16-bit integer type,
        # and a broadcast copies bytes, so this is exact
        dist.broadcast(raw.view(torch.uint8), src=src, group=group)
    return raw


def gather_volume(rec, voxel=None, maxdim=None, group=None, dst=0):
    """Reconstruct this rank's slab of the volume of rec.reconstruct_volume and gather the
    slabs on rank `dst`, which returns (vol tensor [nx, ny, nz], origin, h); the other
    ranks return (None, origin, h)."""
    rank, world = _rank_world(group)
    dims, origin, h = rec._volume_frame(voxel, maxdim)
    nx, ny, nz = dims
    k0, k1 = slab_bounds(nx, rank, world)
    slab, origin, h = rec.reconstruct_volume_slab_tensor(k0, k1, voxel, maxdim)
    if world == 1:
        return slab, origin, h
    # equal-sized messages: pad every slab to the largest one
    cap = -(-nx // world)
    buf = torch.zeros((cap, ny, nz), dtype=slab.dtype, device=slab.device)
    buf[:k1 - k0] = slab
    parts = [torch.empty_like(buf) for _ in range(world)] if rank == dst else None
    dist.gather(buf, parts, dst=dst, group=group)
    if rank != dst:
        return None, origin, h
    vol = torch.empty((nx, ny, nz), dtype=slab.dtype, device=slab.device)
    for r, part in enumerate(parts):
        a, b = slab_bounds(nx, r, world)
        vol[a:b] = part[:b - a]
    return vol, origin, h


def gather_planes(rec, requests, group=None, dst=0):
    """Each rank reconstructs its round-robin share of the slice requests
    (rec.reconstruct_planes_tensor); rank `dst` returns the list of all images in request
    order (f32 tensors [n, n]), the other ranks None."""
    rank, world = _rank_world(group)
    mine = shard_requests(requests, rank, world)
    imgs = rec.reconstruct_planes_tensor([r for _, r in mine]) if mine else []
    if world == 1:
        return list(imgs)
    sizes = [int(r.get("n", 256)) ** 2 for r in requests]
    cap = max(sum(sizes[i] for i in range(len(requests)) if i % world == w) for w in range(world))
    dev = imgs[0].device if len(imgs) else getattr(rec, "device", torch.device("cpu"))
    buf = torch.zeros(max(cap, 1), dtype=torch.float32, device=dev)
    o = 0
    for im in imgs:
        buf[o:o + im.numel()] = im.reshape(-1)
        o += im.numel()
    parts = [torch.empty_like(buf) for _ in range(world)] if rank == dst else None
    dist.gather(buf, parts, dst=dst, group=group)
    if rank != dst:
        return None
    out = [None] * len(requests)
    for w in range(world):
        o = 0
        for i, r in shard_requests(requests, w, world):
            n = int(r.get("n", 256))
            out[i] = parts[w][o:o + n * n].view(n, n)
            o += n * n
    return out
