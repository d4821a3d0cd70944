"""mr_backproject_persistent_noalloc: the persistent back-projection for callers that
cannot call cudaMalloc (their device memory is handed out by another component, or an
allocation on the live acquisition path could synchronise the device). Its work counter
lives in the library's own static device array instead of a caller buffer.

Called through the C ABI, it must give the same images as mr_backproject_persistent with
a caller-owned counter, on two calls in a row with different requests (the shared counter
is re-zeroed by each call), and refuse work lists beyond its fixed scratch. This file is
named to be collected last, so a run that stops at the first failure has already run
every other test; it passes alone in a fresh process as well."""
import numpy as np
import pytest
import torch

from gpu_helpers import DeviceRing
from tomography_local_demo_b200 import _native as N
from tomography_local_demo_b200 import circular_cone_vectors
from tomography_local_demo_b200 import recon as R
from tomography_local_demo_b200.recon import ctypes_void as V

pytestmark = pytest.mark.gpu

A, ROWS, COLS = 48, 40, 56


@pytest.fixture(scope="module")
def ring(cuda):
    geom = circular_cone_vectors(A, 120.0, 200.0, ROWS, COLS, 1.0)
    maps = R.cone_view_maps(R.cone_constants(geom.vectors), ROWS, COLS)
    rng = np.random.default_rng(11)
    q = rng.normal(0, 1, (A, ROWS, COLS)).astype(np.float32)
    return DeviceRing(q, maps, N.MR_CONE, "bf16"), geom.volume_box()


def _batch(box, reqs):
    grids = np.zeros(len(reqs), N.GRID_DTYPE)
    off = 0
    for r, (origin, normal, n, zoom, shift) in enumerate(reqs):
        grids[r] = R.plane_grid(box, origin, normal, n, None, zoom, None, shift)
        grids[r]["out_offset"] = off
        off += n * n
    grids["n_views"] = A
    grids["scale"] = np.pi / A
    return grids, N.plan_tiles(grids), off


def _run(lib, dr, grids, tiles, n_out, noalloc, stream=None):
    """One persistent launch through the C ABI on `stream` (a torch stream, or None for
    the legacy default stream, passed as NULL)."""
    dev = dr.dev
    g_dev = R._struct_tensor(grids, dev)
    t_dev = R._struct_tensor(tiles, dev)
    nt_dev = torch.tensor([len(tiles)], dtype=torch.int64, device=dev)
    out = torch.full((n_out,), float("nan"), dtype=torch.float32, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    if stream is not None:
        stream.wait_stream(torch.cuda.current_stream(dev))
    st = V(stream.cuda_stream) if stream is not None else None
    max_tiles = len(tiles) + 7
    if noalloc:
        rc = lib.mr_backproject_persistent_noalloc(dr.c, V(dr.views.data_ptr()), V(g_dev.data_ptr()),
                                                   V(t_dev.data_ptr()), V(nt_dev.data_ptr()), max_tiles,
                                                   V(out.data_ptr()), V(status.data_ptr()), st)
    else:
        counter = torch.zeros(1, dtype=torch.int32, device=dev)
        rc = lib.mr_backproject_persistent(dr.c, V(dr.views.data_ptr()), V(g_dev.data_ptr()),
                                           V(t_dev.data_ptr()), V(nt_dev.data_ptr()), max_tiles,
                                           V(counter.data_ptr()), V(out.data_ptr()), V(status.data_ptr()), st)
    assert rc == N.MR_OK, lib.mr_status_string(rc)
    torch.cuda.synchronize()
    assert int(status.item()) == 0, "a bounded device-side wait gave up"
    return out.cpu().numpy()


@pytest.mark.parametrize("stream_kind", ["side", "null"])
def test_noalloc_matches_persistent_on_two_calls_in_a_row(ring, stream_kind):
    dr, box = ring
    lib = N.load()
    batches = [
        [((2.0, -1.0, 3.0), (0.4, 0.2, 1.0), 64, 1.0, 0.0), ((0, 0, 0), (1.0, 0.3, 0.1), 96, 2.5, 1.5)],
        [((-3.0, 2.0, 1.0), (0.1, 1.0, 0.4), 128, 1.3, -2.0), ((1, 1, -2), (0.0, 0.0, 1.0), 40, 4.0, 0.0),
         ((0, 2, 0), (0.7, -0.2, 0.5), 72, 1.0, 0.7)],
    ]
    for reqs in batches:
        grids, tiles, n_out = _batch(box, reqs)
        stream = torch.cuda.Stream(dr.dev) if stream_kind == "side" else None
        want = _run(lib, dr, grids, tiles, n_out, noalloc=False, stream=stream)
        got = _run(lib, dr, grids, tiles, n_out, noalloc=True, stream=stream)
        assert np.isfinite(want).all() and np.count_nonzero(want) > 0
        # the same kernel and reduction order: bit-identical, as the server's tests require
        np.testing.assert_array_equal(got, want)


def test_noalloc_rejects_work_beyond_its_scratch(ring):
    dr, _ = ring
    lib = N.load()
    fake = V(1 << 20)          # never dereferenced: the size check fails before any launch
    rc = lib.mr_backproject_persistent_noalloc(dr.c, fake, fake, fake, fake, N.MR_NOALLOC_MAX_TILES + 1,
                                               fake, None, None)
    assert rc == N.MR_ERR_SCRATCH_LIMIT
    assert b"scratch" in lib.mr_status_string(rc)
    assert lib.mr_backproject_persistent_noalloc(dr.c, fake, fake, fake, None, 16, fake, None,
                                                 None) == N.MR_ERR_INVALID


def test_noalloc_rejects_a_stream_of_another_device(ring):
    """The stream's device must be the current device: a stream of another GPU is refused
    on the host before anything is launched (needs two GPUs)."""
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two GPUs")
    dr, box = ring
    lib = N.load()
    grids, tiles, n_out = _batch(box, [((0, 0, 0), (0.0, 0.0, 1.0), 32, 1.0, 0.0)])
    other = (dr.dev.index or 0) + 1
    with torch.cuda.device(other):
        foreign = torch.cuda.Stream(other)
    fake = V(1 << 20)          # never dereferenced: the device check fails before any launch
    with torch.cuda.device(dr.dev):
        rc = lib.mr_backproject_persistent_noalloc(dr.c, fake, fake, fake, fake, len(tiles), fake, None,
                                                   V(foreign.cuda_stream))
    assert rc == N.MR_ERR_INVALID
