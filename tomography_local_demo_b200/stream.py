"""Simulated live acquisition (minirecast stream.py:1-64): push projections into any
sink with add_projections(indices, block), in sequential or bit-reversed order."""
import threading
import time

import numpy as np


def arrival_order(n, mode="sequential"):
    """Acquisition order of n views: "sequential" 0..n-1, or "interleaved" = bit-reversed
    indices (every group spreads evenly over the full angular range)."""
    if mode == "sequential":
        return np.arange(n)
    if mode == "interleaved":
        bits = max(1, int(np.ceil(np.log2(n))))
        idx = np.arange(1 << bits)
        rev = np.zeros_like(idx)
        for b in range(bits):
            rev |= ((idx >> b) & 1) << (bits - 1 - b)
        return rev[rev < n]
    raise ValueError(f"unknown order {mode!r}")


class Feeder(threading.Thread):
    """Push `proj` ([rows, angles, cols]) into `sink` at `rate` projections/s
    (rate <= 0: as fast as the sink accepts)."""

    def __init__(self, sink, proj, order="sequential", group=20, rate=100.0, verbose=True):
        super().__init__(daemon=True)
        self.sink = sink
        self.proj = proj
        self.order = arrival_order(proj.shape[1], order)
        self.group = max(1, int(group))
        self.rate = float(rate)
        self.verbose = verbose
        self.stop_event = threading.Event()
        self.sent = 0

    def run(self):
        t0 = time.perf_counter()
        for i in range(0, len(self.order), self.group):
            if self.stop_event.is_set():
                return
            idx = self.order[i:i + self.group]
            self.sink.add_projections(idx, np.ascontiguousarray(self.proj[:, idx, :]))
            self.sent = i + len(idx)
            if self.rate > 0:
                wait = t0 + self.sent / self.rate - time.perf_counter()
                if wait > 0:
                    self.stop_event.wait(wait)
        if self.verbose:
            dt = time.perf_counter() - t0
            print(f"[stream] {self.sent} projections streamed in {dt:.1f}s "
                  f"({self.sent / max(dt, 1e-9):.0f}/s)")

    def stop(self):
        self.stop_event.set()
