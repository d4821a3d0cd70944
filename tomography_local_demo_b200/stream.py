"""Simulated live acquisition: views of a scan become due on a schedule and are pushed
into a sink, any object with add_projections(indices, block) (a SliceReconstructor, a
net.RemoteSink, a SliceServer's reconstructor).

The contract is minirecast's (stream.py:12-64): views arrive in sequential or
bit-reversed order, in groups of `group`, at `rate` views per second (rate <= 0: as fast
as the sink takes them), the first group at once and each next group when the views
already sent are due. Here the timing is an `AcquisitionSchedule` - a plain list of
(due time, view indices) - that the threaded `Feeder` and the bench's serving simulation
both follow.
"""
import threading
import time

import numpy as np


def arrival_order(n, mode="sequential"):
    """Acquisition order of n views.

    "sequential"  : 0, 1, ..., n-1 (a continuous rotation);
    "interleaved" : the bit-reversal permutation of 0 .. 2^b - 1 (b = max(1, ceil(log2 n)))
                    with the indices >= n dropped, so that every run of consecutive
                    arrivals spreads over the whole angular range. The order must be the
                    reference's (stream.py:12-29), or a streamed scan would see other view
                    subsets at each point in time.
    """
    if mode == "sequential":
        return np.arange(n)
    if mode == "interleaved":
        bits = max(1, (int(n) - 1).bit_length())
        # van der Corput construction: the bit-reversal permutation of 2^(b+1) indices is
        # that of 2^b indices doubled, followed by the same plus one
        perm = np.zeros(1, dtype=np.int64)
        for _ in range(bits):
            perm = np.concatenate([2 * perm, 2 * perm + 1])
        return perm[perm < n]
    raise ValueError(f"unknown order {mode!r}")


class AcquisitionSchedule:
    """When each group of a scan's views is due.

    The scan's `n` views are taken in `arrival_order(n, order)` and cut into groups of
    `group`; group k is due `sent_k / rate` seconds after the start, sent_k being the
    number of views in groups 0 .. k-1 (all due at 0 when rate <= 0). Iterating yields
    (due_seconds, indices) pairs."""

    def __init__(self, n, order="sequential", group=20, rate=100.0):
        self.order = arrival_order(n, order) if isinstance(order, str) else np.asarray(order)
        self.group = max(1, int(group))
        self.rate = float(rate)
        starts = np.arange(0, len(self.order), self.group)
        self.groups = [self.order[s:s + self.group] for s in starts]
        self.due = starts / self.rate if self.rate > 0 else np.zeros(len(starts))

    def __len__(self):
        return len(self.groups)

    def __iter__(self):
        return iter(zip(self.due.tolist(), self.groups))

    def due_by(self, elapsed):
        """Number of groups due `elapsed` seconds after the start."""
        return int(np.searchsorted(self.due, elapsed, side="right"))


class Feeder(threading.Thread):
    """Push the projections `proj` ([rows, angles, cols], a NumPy array or a torch tensor)
    into `sink` on an AcquisitionSchedule, from its own thread (start / join / stop) or
    from the caller's (run).

    `sent` counts the views pushed so far; stop() ends the feed before the next group."""

    def __init__(self, sink, proj, order="sequential", group=20, rate=100.0, verbose=True):
        super().__init__(daemon=True, name="minirecast-feeder")
        self.sink = sink
        self.proj = proj
        self.schedule = AcquisitionSchedule(proj.shape[1], order, group, rate)
        self.order = self.schedule.order
        self.group, self.rate = self.schedule.group, self.schedule.rate
        self.verbose = verbose
        self.sent = 0
        self._halt = threading.Event()

    def _block(self, idx):
        blk = self.proj[:, idx, :]
        return np.ascontiguousarray(blk) if isinstance(blk, np.ndarray) else blk.contiguous()

    def run(self):
        start = time.perf_counter()
        for due, idx in self.schedule:
            # sleep until the group is due; a stop() during the sleep ends the feed
            if self._halt.wait(max(0.0, start + due - time.perf_counter())):
                return
            self.sink.add_projections(idx, self._block(idx))
            self.sent += len(idx)
        if self.verbose:
            took = time.perf_counter() - start
            print(f"[stream] pushed {self.sent} views in {took:.1f} s "
                  f"({self.sent / max(took, 1e-9):.0f} views/s)")

    def stop(self):
        self._halt.set()

    @property
    def stopped(self):
        return self._halt.is_set()
