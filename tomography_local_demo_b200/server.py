"""Device-resident, continuously batched slice server (the request loop of minirecast
net.py:129-154 - "slice", "preview" - rebuilt around one GPU).

    srv = SliceServer(rec, budget_bytes=20e9)
    fut = srv.submit(origin, normal, n=512, zoom=2.0, cor_shift=1.5)   # -> Future
    img = fut.result()                                                # f32 [n, n]

* Requests of any size, zoom, orientation and COR offset queue up; the dispatcher
  admits them in arrival order while their output bytes fit the memory budget and a
  batch slot is free, and sends each admitted batch to the GPU as ONE launch of the
  persistent back-projector (mr_backproject_persistent): a fixed grid of CTA clusters
  that pulls tiles of every request in the batch from a device work counter.
* That launch is captured once per batch slot in a CUDA graph and replayed; per batch
  only the request descriptors are copied (pinned host -> device) before the replay and
  the images (device -> pinned host) after it.
* Two batch slots on two streams: while one batch runs, the next is admitted and
  launched, so their work overlaps on the device; new projections are filtered on the
  reconstructor's own ingest stream meanwhile (add_projections / add_raw_projections).
* Each request sees the views received when its batch was admitted (snapshot); the
  per-tile arithmetic and the cluster reduction order do not depend on the batch, so a
  result is bit-identical alone and in any mix.
Latencies (submit -> result on the host) are kept in `latencies` (request kinds in
`latency_kinds`).
"""
import collections
import threading
import time
from concurrent.futures import Future

import numpy as np
import torch

from . import _native as N
from .recon import ctypes_void, plane_grid, volume_grid_record


class _Req:
    __slots__ = ("grid", "nbytes", "shape", "future", "t_submit", "kind", "meta")

    def __init__(self, grid, shape, kind, meta=None):
        self.grid = grid
        self.shape = shape
        self.nbytes = int(np.prod(shape)) * 4
        self.future = Future()
        self.t_submit = time.perf_counter()
        self.kind = kind
        self.meta = meta


class _Slot:
    """Device/pinned buffers, stream and captured graph of one in-flight batch."""

    def __init__(self, dev, max_grids, max_tiles, pool_floats):
        self.stream = torch.cuda.Stream(dev)
        with torch.cuda.device(dev):
            self.grids_dev = torch.zeros(max_grids * N.GRID_DTYPE.itemsize, dtype=torch.uint8, device=dev)
            self.tiles_dev = torch.zeros(max_tiles * N.TILE_DTYPE.itemsize, dtype=torch.uint8, device=dev)
            self.ntiles_dev = torch.zeros(1, dtype=torch.int64, device=dev)
            self.counter = torch.zeros(1, dtype=torch.int32, device=dev)     # 4-byte work counter
            self.status = torch.zeros(1, dtype=torch.int32, device=dev)
            self.out = torch.zeros(pool_floats, dtype=torch.float32, device=dev)
        self.grids_host = torch.zeros(max_grids * N.GRID_DTYPE.itemsize, dtype=torch.uint8).pin_memory()
        self.tiles_host = torch.zeros(max_tiles * N.TILE_DTYPE.itemsize, dtype=torch.uint8).pin_memory()
        self.ntiles_host = torch.zeros(1, dtype=torch.int64).pin_memory()
        self.out_host = torch.zeros(pool_floats, dtype=torch.float32).pin_memory()
        self.graph = None
        self.done = torch.cuda.Event()
        self.busy = False


class SliceServer:
    def __init__(self, rec, budget_bytes=20e9, max_batch=64, max_tiles=1 << 16, pool_bytes=256 << 20,
                 slots=2, use_graphs=True):
        self.rec = rec
        self.dev = rec.device
        self.budget = int(budget_bytes)
        self.max_batch = int(max_batch)
        self.max_tiles = int(max_tiles)
        self.pool_floats = int(pool_bytes) // 4
        self.use_graphs = use_graphs
        self.slots = [_Slot(self.dev, self.max_batch, self.max_tiles, self.pool_floats) for _ in range(slots)]
        if use_graphs:
            # every slot's graph is captured here, before the first request: a capture
            # synchronises the device and collects the interpreter's garbage, a pause of
            # tens of milliseconds that would otherwise land on whichever request first
            # reaches each slot
            for slot in self.slots:
                self._capture(slot)
        self.queue = collections.deque()
        self.cv = threading.Condition()
        self.in_flight = 0
        self.latencies = []
        self.latency_kinds = []
        self.batches = 0
        self.updates = 0
        self._running = True
        self._completions = collections.deque()
        self._ccv = threading.Condition()
        self._dispatcher = threading.Thread(target=self._dispatch_loop, daemon=True)
        self._completer = threading.Thread(target=self._complete_loop, daemon=True)
        self._dispatcher.start()
        self._completer.start()

    # ------------------------------------------------------------------ client side
    def submit(self, origin, normal, n=256, size=None, zoom=1.0, center=None, cor_shift=None):
        """Queue one slice; the Future resolves to an f32 [n, n] image (0 outside the box)."""
        shift = self.rec.cor_shift if cor_shift is None else float(cor_shift)
        g = plane_grid(self.rec.box, origin, normal, int(n), size, zoom, center, shift)
        return self._enqueue(_Req(g, (int(n), int(n)), "slice"))

    def submit_preview(self, maxdim=128):
        """Queue a low-resolution volume of the whole box (preview_volume, recon.py:472-475);
        the Future resolves to (f32 [nx, ny, nz], origin, voxel size)."""
        dims, origin, h = self.rec._volume_frame(None, maxdim)
        g = volume_grid_record(origin, h, dims)
        g["cor_shift"] = self.rec.cor_shift
        return self._enqueue(_Req(g, tuple(dims), "volume", (origin, h)))

    def _enqueue(self, req):
        if req.nbytes > min(self.budget, self.pool_floats * 4):
            req.future.set_exception(MemoryError(f"request of {req.nbytes} bytes exceeds the admission "
                                                 f"budget / batch pool"))
            return req.future
        with self.cv:
            self.queue.append(req)
            self.cv.notify_all()
        return req.future

    def close(self):
        with self.cv:
            self._running = False
            self.cv.notify_all()
        self._dispatcher.join(5)
        with self._ccv:
            self._ccv.notify_all()
        self._completer.join(5)

    def device_status(self):
        """Raise TimeoutError if a bounded device-side wait of any batch gave up."""
        for s in self.slots:
            s.stream.synchronize()
            code = int(s.status.item())
            if code != 0:
                N.check(code, "slice server batch")

    def stats(self):
        """Request count, batches, updates and latency percentiles (ms) over all requests,
        and over the slice requests alone (previews are volumes, far larger requests)."""
        n = min(len(self.latencies), len(self.latency_kinds))     # the completer may be mid-append
        lat = np.array(self.latencies[:n]) * 1e3
        sl = lat[np.array(self.latency_kinds[:n]) == "slice"] if n else lat
        pct = lambda a, q: float(np.percentile(a, q)) if len(a) else None     # noqa: E731
        return {"requests": len(lat), "batches": self.batches, "updates": self.updates,
                "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99),
                "slice_p50_ms": pct(sl, 50), "slice_p99_ms": pct(sl, 99)}

    # ------------------------------------------------------------------ device side
    def _free_slot(self):
        for s in self.slots:
            if not s.busy:
                return s
        return None

    def _dispatch_loop(self):
        while True:
            with self.cv:
                while self._running and (not self.queue or self._free_slot() is None):
                    self.cv.wait(0.05)
                if not self._running:
                    return
                slot = self._free_slot()
                batch, used, tiles_est = [], 0, 0
                while self.queue and len(batch) < self.max_batch:
                    r = self.queue[0]
                    if self.in_flight + used + r.nbytes > self.budget or used + r.nbytes > self.pool_floats * 4:
                        break
                    batch.append(self.queue.popleft())
                    used += r.nbytes
                if not batch:
                    continue
                self.in_flight += used
                slot.busy = True
            try:
                self._launch(slot, batch)
            except Exception as e:                        # fail the batch, keep serving
                with self.cv:
                    self.in_flight -= used
                    slot.busy = False
                    self.cv.notify_all()
                for r in batch:
                    r.future.set_exception(e)

    def _capture(self, slot):
        """Capture the slot's persistent launch in a CUDA graph (on the slot's stream). The
        launch reads its batch from the slot's device buffers, so one graph serves every
        batch the slot takes."""
        with torch.cuda.device(self.dev), torch.cuda.stream(slot.stream):
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=slot.stream, capture_error_mode="thread_local"):
                self._graph_launch(slot)
        slot.graph = g

    def _graph_launch(self, slot):
        rec = self.rec
        v = ctypes_void
        N.check(N.load().mr_backproject_persistent(
            rec._ring_c, v(rec._views_dev.data_ptr()), v(slot.grids_dev.data_ptr()), v(slot.tiles_dev.data_ptr()),
            v(slot.ntiles_dev.data_ptr()), self.max_tiles, v(slot.counter.data_ptr()), v(slot.out.data_ptr()),
            v(slot.status.data_ptr()), v(torch.cuda.current_stream(self.dev).cuda_stream)),
            "mr_backproject_persistent")

    def _launch(self, slot, batch):
        rec = self.rec
        n_views, _, ev = rec._snapshot()
        grids = np.zeros(len(batch), dtype=N.GRID_DTYPE)
        off = 0
        for i, r in enumerate(batch):
            grids[i] = r.grid
            grids[i]["out_offset"] = off
            off += int(np.prod(r.shape))
        grids["n_views"] = n_views
        grids["scale"] = np.pi / n_views if n_views else 0.0
        tiles = N.plan_tiles(grids, getattr(rec, "_band_axis", None))
        if len(tiles) > self.max_tiles:
            raise MemoryError(f"batch needs {len(tiles)} tiles > {self.max_tiles}")
        st = slot.stream
        with torch.cuda.device(self.dev), torch.cuda.stream(st):
            if ev is not None:
                st.wait_event(ev)
            gb = np.ascontiguousarray(grids).view(np.uint8)
            tb = np.ascontiguousarray(tiles).view(np.uint8)
            slot.grids_host[:gb.size].numpy()[:] = gb
            slot.tiles_host[:tb.size].numpy()[:] = tb
            slot.ntiles_host[0] = len(tiles)
            slot.grids_dev[:gb.size].copy_(slot.grids_host[:gb.size], non_blocking=True)
            if tb.size:
                slot.tiles_dev[:tb.size].copy_(slot.tiles_host[:tb.size], non_blocking=True)
            slot.ntiles_dev.copy_(slot.ntiles_host, non_blocking=True)
            if n_views > 0 and len(tiles) > 0:
                if self.use_graphs:
                    if slot.graph is None:
                        self._capture(slot)
                    slot.graph.replay()
                else:
                    self._graph_launch(slot)
            else:
                slot.out[:off].zero_()
            slot.out_host[:off].copy_(slot.out[:off], non_blocking=True)
            slot.done.record(st)
        self.batches += 1
        with self._ccv:
            self._completions.append((slot, batch, off, n_views, grids))
            self._ccv.notify_all()

    def _complete_loop(self):
        while True:
            with self._ccv:
                while not self._completions and self._running:
                    self._ccv.wait(0.05)
                if not self._completions:
                    if not self._running:
                        return
                    continue
                slot, batch, off, n_views, grids = self._completions.popleft()
            slot.done.synchronize()
            host = slot.out_host[:off].numpy()
            t = time.perf_counter()
            o = 0
            res = []
            for r in batch:
                sz = int(np.prod(r.shape))
                img = host[o:o + sz].reshape(r.shape).copy()
                o += sz
                res.append(img)
            used = sum(r.nbytes for r in batch)
            with self.cv:
                self.in_flight -= used
                slot.busy = False
                self.cv.notify_all()
            for r, img in zip(batch, res):
                self.latencies.append(t - r.t_submit)
                self.latency_kinds.append(r.kind)
                if r.kind == "slice":
                    self.updates += int(np.count_nonzero(img)) * n_views
                    r.future.set_result(img)
                else:
                    origin, h = r.meta
                    self.updates += img.size * n_views
                    r.future.set_result((img, origin, h))
