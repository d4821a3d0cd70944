#!/usr/bin/env python
"""Benchmark of the cone-beam FDK hot path on B200.

Workload (one step): a cone-beam scan of 600 views (486 x 384 detector, 0.299 mm,
SOD 440 / SDD 680 mm, 40 seeded random ellipsoids in a 60 mm sphere, raw uint16 counts
with flat ~ 50000 +/- 2 %, dark ~ 100 +/- 5 and Poisson noise) is ingested - fused
correction, -log, FDK weight and ramp filter into the device ring - and three
arbitrarily oriented 512 x 512 slices (seeded random unit normals, offsets within
+/-10 mm) are back-projected from all 600 views in one batched launch.

Metric: voxel-projection updates/s = (in-box slice pixels x views) / step time.
  value : device time with the raw counts already resident in HBM (CUDA events), the
          step replayed from a captured CUDA graph (SliceReconstructor.scan_replay); the
          same step issued eagerly through the public calls is reported under "eager"
  e2e   : the public API with pinned host buffers (H2D of the raw counts, D2H of the
          three images inside the timed region), host wall clock
Multi-GPU (torchrun): every rank runs its own scan (independent objects, no
collective on the data path); value = all ranks' updates / max-over-ranks time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import ctypes
import gc
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(views=600, rows=384, cols=486, pixel=0.299, sod=440.0, sdd=680.0,
                ellipsoids=40, phantom_seed=2, noise_seed=7, slice_seed=11, slices=3, n=512)
WORKLOAD_NAME = ("cone FDK: 600 raw uint16 views 486x384 -> filtered ring -> "
                 "3 oblique 512x512 slices in one batched launch")
FP32_LANE_OPS_PER_UPDATE = 26       # algorithmic FP32 operations per voxel-projection update
NOMINAL_FP32_LANE_OPS = 148 * 128 * 1965e6   # SMs x FP32 lanes x max SM clock (ops/s)


# ------------------------------------------------------------------ workload
def geometry():
    from tomography_local_demo_b200 import circular_cone_vectors
    w = WORKLOAD
    return circular_cone_vectors(w["views"], w["sod"], w["sdd"], w["rows"], w["cols"], w["pixel"])


def slice_requests(box):
    rng = np.random.default_rng(WORKLOAD["slice_seed"])
    reqs = []
    for _ in range(WORKLOAD["slices"]):
        nrm = rng.normal(size=3)
        nrm /= np.linalg.norm(nrm)
        reqs.append(dict(origin=tuple(rng.uniform(-10, 10) * nrm), normal=tuple(nrm), n=WORKLOAD["n"]))
    return reqs


def in_box_pixels(box, reqs):
    from tomography_local_demo_b200.recon import slice_points
    return [int(slice_points(box, r["origin"], r["normal"], r["n"])[1].sum()) for r in reqs]


def make_scan(device):
    """Raw uint16 counts [views, rows, cols] + flat/dark frames, synthesised on `device`."""
    import torch
    from tomography_local_demo_b200 import phantom as PH
    w = WORKLOAD
    geom = geometry()
    ph = PH.EllipsoidPhantom(1.0, PH.random_ellipsoids(w["ellipsoids"], w["phantom_seed"]))
    p = PH.project_cone_torch(ph, geom, device=device)
    gen = torch.Generator(device=device)
    gen.manual_seed(w["noise_seed"])
    shape = (w["rows"], w["cols"])
    flat = 50000.0 * (1.0 + 0.02 * torch.randn(shape, generator=gen, device=device, dtype=torch.float64))
    dark = 100.0 + 5.0 * torch.randn(shape, generator=gen, device=device, dtype=torch.float64)
    raw = PH.raw_counts(p, flat, dark, seed=w["noise_seed"])
    flats = torch.stack([torch.poisson((flat - dark).clamp(min=0), generator=gen) + dark for _ in range(4)])
    darks = torch.stack([dark + torch.randn(shape, generator=gen, device=device, dtype=torch.float64)
                         for _ in range(4)])
    u16 = lambda t: t.round().clamp(0, 65535).to(torch.int32).to(torch.int16)  # noqa: E731 (uint16 bits)
    return geom, raw.to(torch.int16), u16(flats), u16(darks)


def as_u16(t):
    return t.cpu().numpy().view(np.uint16)


# ------------------------------------------------------------------ clocks
def _clock_sampler_process(conn, uuid, index, period):
    """Child process of ClockSampler: NVML samples (monotonic time, SM MHz, clock-event
    reasons, W) every `period` s until told to stop, then all of them (read-only queries)."""
    samples = []
    try:
        import pynvml as nv
        nv.nvmlInit()
        try:
            h = nv.nvmlDeviceGetHandleByUUID(uuid.encode()) if uuid else nv.nvmlDeviceGetHandleByIndex(index)
        except Exception:
            h = nv.nvmlDeviceGetHandleByIndex(index)
        reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        conn.send(("ready", float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))))
        while True:
            samples.append((time.monotonic(), float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                            int(reasons(h)), nv.nvmlDeviceGetPowerUsage(h) / 1e3))
            if conn.poll(period):
                conn.recv()
                samples.append((time.monotonic(), float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                int(reasons(h)), nv.nvmlDeviceGetPowerUsage(h) / 1e3))
                break
        conn.send(("samples", samples))
    except Exception as e:                 # no NVML: report unsampled
        conn.send(("error", repr(e)))


class ClockSampler:
    """Samples SM clock, power and clock-event reasons every 2 ms through NVML (read-only
    queries; nothing is set) in a child process, and keeps the samples of the timed region
    (from mark() to the end, plus one right after it). A process of its own: NVML queries
    in the benchmarking process held up its CUDA calls (its first queries take ~0.85 ms
    each) and a sampling thread competes for the interpreter."""
    BITS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
            "sw_power_cap": 0x4}

    def __init__(self, device_index):
        self.dev = device_index
        self.samples = []
        self.max_mhz = None
        self.error = None
        self._proc = None
        self._t0 = None

    def __enter__(self):
        import multiprocessing as mp
        import torch
        uuid = None
        try:
            uuid = "GPU-" + str(torch.cuda.get_device_properties(self.dev).uuid)
        except Exception:
            pass
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        index = int(vis.split(",")[self.dev]) if vis and vis.split(",")[0].isdigit() else self.dev
        try:
            ctx = mp.get_context("spawn")
            self._conn, child = ctx.Pipe()
            self._proc = ctx.Process(target=_clock_sampler_process, args=(child, uuid, index, 0.002), daemon=True)
            self._proc.start()
            if self._conn.poll(60):
                kind, val = self._conn.recv()
                if kind == "ready":
                    self.max_mhz = val
                else:
                    self.error = val
            else:
                self.error = "clock sampler did not start"
        except Exception as e:
            self.error = repr(e)
        return self

    def mark(self):
        """Start of the timed region (samples before it are dropped)."""
        self._t0 = time.monotonic()

    def __exit__(self, *a):
        t1 = time.monotonic()
        if self._proc is None or self.max_mhz is None:
            return
        try:
            self._conn.send("stop")
            if self._conn.poll(30):
                kind, val = self._conn.recv()
                if kind == "samples":
                    t0 = self._t0 if self._t0 is not None else t1
                    inside = [x for x in val if t0 <= x[0] <= t1]
                    after = [x for x in val if x[0] > t1][:1]
                    self.samples = [x[1:] for x in inside + after]
                else:
                    self.error = val
        except Exception as e:
            self.error = repr(e)
        finally:
            self._proc.join(10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"],
                    "error": self.error}
        reasons = sorted({k for _, r, _ in self.samples for k, bit in self.BITS.items() if r & bit})
        return {"sm_mhz": float(np.median([c for c, _, _ in self.samples])), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.samples),
                "power_w_max": float(max(p for _, _, p in self.samples))}


# ------------------------------------------------------------------ distributed
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl"
        import torch
        if not torch.cuda.is_available():
            backend = "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world, device=None):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------------ CPU legs (oracle)
def cpu_job(raw_u16, flats_u16, darks_u16, geom, reqs, box, precision="ref", threads=None):
    """The reference's CPU algorithm (oracle port): correction, FDK filter, then every
    in-box pixel of the slices back-projected from all views.
    Returns ([(mask, values) per slice], timings dict)."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import bp as obp
    from oracle import filter as of
    threads = threads or os.cpu_count()
    obp.threads(threads)
    A = raw_u16.shape[0]
    t0 = time.perf_counter()
    d_b = np.mean([of.bin_mean(f, 1) for f in darks_u16], axis=0)
    f_b = np.mean([of.bin_mean(f, 1) for f in flats_u16], axis=0)
    gain = (1.0 / np.maximum(f_b - d_b, 1.0)).astype(np.float32)
    K = of.cone_constants(geom.vectors)
    exact = precision == "fp64"

    def chunk(i0):
        i1 = min(A, i0 + 16)
        x = -np.log(np.clip((raw_u16[i0:i1].astype(np.float32) - d_b) * gain, 1e-3, None))
        Kc = {k: v[i0:i1] for k, v in K.items()}
        return i0, of.fdk_filter_block(np.transpose(x, (1, 0, 2)), Kc, "shepp-logan", exact64=exact)

    q = np.zeros((A,) + raw_u16.shape[1:], np.float64 if exact else np.float32)
    with ThreadPoolExecutor(threads) as ex:
        for i0, part in ex.map(chunk, range(0, A, 16)):
            q[i0:i0 + len(part)] = part
    t_filter = time.perf_counter() - t0
    from oracle import geometry as og
    vals, n_upd, t_bp = [], 0, 0.0
    for r in reqs:
        pts, sel = og.slice_points(box, r["origin"], r["normal"], r["n"])
        P = pts[sel]
        t1 = time.perf_counter()
        v = obp.bp_cone(q[:A], K["s"][:A], K["d"][:A], K["uu"][:A], K["vv"][:A], K["n"][:A],
                        K["sdd"][:A], K["sod"][:A], P, np.pi / A)
        t_bp += time.perf_counter() - t1
        n_upd += len(P) * A
        vals.append((sel, v))
    return vals, dict(t_filter=t_filter, views=A, t_bp=t_bp, updates=n_upd, threads=threads)


# ------------------------------------------------------------------ our arm
def run_ours(args, rank, world, local):
    import torch
    from tomography_local_demo_b200 import SliceReconstructor
    from tomography_local_demo_b200.recon import KernelTimer
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    clocks = ClockSampler(local).__enter__()      # sampling from set-up on (see mark())
    geom, raw_dev, flats, darks = make_scan(dev)
    box = geom.volume_box()
    reqs = slice_requests(box)
    inbox = in_box_pixels(box, reqs)
    V = WORKLOAD["views"]
    updates = sum(inbox) * V
    idx = np.arange(V)

    rec = SliceReconstructor(None, geom, store=args.store, verbose=False, device=dev, filter=args.filter)
    rec.set_flat_dark(as_u16(flats), as_u16(darks))
    timer = KernelTimer()

    def step_device():
        rec.reset()
        rec.add_raw_projections(idx, raw_dev)
        return rec.reconstruct_planes_tensor(reqs)

    for _ in range(args.warmup):
        step_device()
    torch.cuda.synchronize()
    barrier(world)
    rec.kernel_timer = timer
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    # the interpreter's cyclic garbage collector stays off inside the timed regions (as in
    # timeit): a full collection is a pause of the launching thread unrelated to the path
    gc.collect()
    gc.disable()
    clocks.mark()
    e0.record(rec.ingest_stream)
    h0 = time.perf_counter()
    for _ in range(args.steps):
        step_device()
    t_issue = time.perf_counter() - h0         # host time to issue the steps (the GPU may still run)
    e1.record(rec.stream)
    torch.cuda.synchronize()
    gc.enable()
    barrier(world)
    rec.kernel_timer = None
    t_eager = max_over_ranks(e0.elapsed_time(e1) / 1e3, world, dev)
    kern = timer.summary()

    # ---- the same step replayed from a captured CUDA graph (ScanReplay: the ingest and
    # the batched back-projection, no host work between steps); this is the device
    # throughput, free of the host's issue time, which the eager loop above exposes when
    # the host is slower than the device
    value_source = "graph replay (SliceReconstructor.scan_replay)"
    try:
        replay = rec.scan_replay(raw_dev, reqs)
    except RuntimeError as e:               # a capture refused by this driver / runtime
        replay, value_source = None, f"eager step (graph capture failed: {str(e)[:120]})"
    if replay is not None:
        for _ in range(args.warmup):
            replay.replay()
    torch.cuda.synchronize()
    barrier(world)
    if replay is not None:
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(replay.stream)
        for _ in range(args.steps):
            replay.replay()
        g1.record(replay.stream)
    torch.cuda.synchronize()
    clocks.__exit__(None, None, None)
    barrier(world)
    if replay is not None:
        t_dev = max_over_ranks(g0.elapsed_time(g1) / 1e3, world, dev)
        launches = 2 * args.steps             # one ingest and one back-projection per replay
    else:
        t_dev = t_eager
        launches = sum(n for n, _ in kern.values())
    del replay

    # ---- end to end through the public API, pinned host buffers
    raw_host = torch.empty(raw_dev.shape, dtype=torch.int16, pin_memory=True)
    raw_host.copy_(raw_dev)
    rec_e = SliceReconstructor(None, geom, store=args.store, verbose=False, device=dev, filter=args.filter)
    rec_e.set_flat_dark(as_u16(flats), as_u16(darks))

    def step_e2e():
        rec_e.reset()
        rec_e.add_raw_projections(idx, raw_host)
        return rec_e.reconstruct_planes(reqs)

    for _ in range(args.warmup):
        step_e2e()
    torch.cuda.synchronize()
    barrier(world)
    gc.collect()
    gc.disable()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step_e2e()
    torch.cuda.synchronize()
    t_e2e_local = time.perf_counter() - t0
    gc.enable()
    t_e2e = max_over_ranks(t_e2e_local, world, dev)
    h2d = raw_host.numel() * 2 + V * (64 + 32) + len(reqs) * 256
    d2h = sum(r["n"] ** 2 for r in reqs) * 8         # the images come back as float64

    # ---- back-projection only: bf16 batched vs plain fp32 one request per launch
    extra = {}
    if rank == 0:
        extra = bp_only_and_latency(args, dev, geom, raw_dev, flats, darks, reqs, updates, rec)

    if rank != 0:
        return None
    ms = t_dev / args.steps * 1e3
    value = updates * world * args.steps / t_dev
    # roofline of the dominant kernel (largest share of device time in the timed region)
    dom = max(kern.items(), key=lambda kv: kv[1][1])
    line = {
        "metric": "voxel-proj updates/s", "value": value, "unit": "updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD_NAME, "views": V, "rows": WORKLOAD["rows"],
                   "cols": WORKLOAD["cols"], "slices": len(reqs), "n": WORKLOAD["n"],
                   "in_box_pixels": inbox, "store": args.store, "filter": args.filter, "accumulate": "f32",
                   "parallelism": f"replicas x{world}",
                   "l2": "no flush: every step reads 224 MB raw counts and writes/reads the "
                         f"{'224' if args.store != 'fp32' else '448'} MB ring (> 126 MB L2)"},
        "e2e": {"value": updates * world * args.steps / t_e2e, "unit": "updates/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": t_e2e / args.steps * 1e3},
        "value_source": value_source,
        "eager": {"ms_per_step": t_eager / args.steps * 1e3, "host_issue_ms_per_step": t_issue / args.steps * 1e3,
                  "note": "the same step through reset / add_raw_projections / reconstruct_planes_tensor, "
                          "issued from the host each step; its launches give the per-kernel times"},
        "gpu_launches": launches,
        "kernels": {k: {"launches": n, "avg_ms": t / n, "share": t / sum(x[1] for x in kern.values())}
                    for k, (n, t) in kern.items()},
        "clocks": clocks.summary(),
    }
    line["roofline"] = roofline(dom[0], dom[1], updates, args.store)
    other = [k for k in kern if k != dom[0]]
    if other:
        line["roofline_" + other[0]] = roofline(other[0], kern[other[0]], updates, args.store)
    imgs = extra.pop("_images", None)
    line.update(extra)
    if rank == 0 and not args.no_serve:
        line["serving"] = serving_simulation(args, dev, geom, raw_dev, flats, darks)
        line["serving_fp32_one_request_per_launch"] = serving_simulation(args, dev, geom, raw_dev, flats, darks,
                                                                         store="fp32", max_batch=1)
    if world == 1 and not args.no_cpu:
        line["cpu_baseline"], line["accuracy"] = cpu_baseline_and_accuracy(
            args, geom, raw_dev, flats, darks, reqs, box, updates, imgs)
    return line


def _traffic(kernel):
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get(kernel, {}).get("dram_bytes_per_launch")
    except (OSError, ValueError):
        return None


def roofline(name, stats, updates, store):
    from tomography_local_demo_b200.recon import ring_pitch
    n, t_ms = stats
    avg = t_ms / n / 1e3
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except (OSError, ValueError):
        pass
    if name == "mr_ingest_u16_tc":
        # tensor-core Toeplitz filter: MMA flops executed per launch (x_hi g_hi over the
        # 64-padded row, plus the two cross terms on the near block diagonals)
        w = WORKLOAD
        kb = (w["cols"] + 63) // 64
        tiles = -(-w["views"] * w["rows"] // 128)
        near = sum(64 * (min(kb - 1, i + 1) - max(0, i - 1) + 1) for i in range(kb))
        flops = tiles * (kb * 2 * 128 * 64 * (64 * kb) + 2 * 2 * 128 * 64 * near)
        peak = peaks.get("bf16_tflops", 1590.0)
        ach = flops / avg / 1e12
        out_b = 2 if store != "fp32" else 4
        pitch = ring_pitch(w["cols"], store)
        alg_bytes = w["views"] * w["rows"] * (w["cols"] * 2 + pitch * out_b)
        return {"kernel": name, "bound": "tensor", "achieved": ach, "peak": peak, "unit": "TFLOP/s",
                "frac": ach / peak, "traffic": _traffic(name), "executed_flops": flops,
                "dense_toeplitz_flops": 2 * w["views"] * w["rows"] * w["cols"] ** 2,
                "hbm_gbs": alg_bytes / avg / 1e9, "hbm_frac": alg_bytes / avg / 1e9 / peaks.get("hbm_gbs", 6650.0),
                "peak_source": "measured dense bf16 (the f16 kind runs at the same rate)" if "bf16_tflops" in peaks
                else "fallback"}
    if name == "mr_ingest_u16":
        w = WORKLOAD
        out_b = 2 if store != "fp32" else 4
        pitch = ring_pitch(w["cols"], store)
        alg = w["views"] * w["rows"] * (w["cols"] * 2 + pitch * out_b)
        peak = peaks.get("hbm_gbs", 6650.0)
        ach = alg / avg / 1e9
        return {"kernel": name, "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": ach / peak, "traffic": _traffic(name), "algorithmic_bytes": alg,
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"}
    ops = updates * FP32_LANE_OPS_PER_UPDATE
    ach = ops / avg / 1e12
    peak = NOMINAL_FP32_LANE_OPS / 1e12
    return {"kernel": name, "bound": "fp32-issue", "achieved": ach, "peak": peak,
            "unit": "T FP32-lane-ops/s", "frac": ach / peak, "traffic": _traffic(name),
            "algorithmic_ops": ops, "updates_per_s": updates / avg,
            "peak_source": "nominal (148 SMs x 128 FP32 lanes x 1965 MHz); not in MEASURED_PEAKS.json"}


def bp_only_and_latency(args, dev, geom, raw_dev, flats, darks, reqs, updates, rec_bf16):
    import torch
    from tomography_local_demo_b200 import SliceReconstructor
    V = WORKLOAD["views"]
    idx = np.arange(V)
    rec32 = SliceReconstructor(None, geom, store="fp32", verbose=False, device=dev)
    rec32.set_flat_dark(as_u16(flats), as_u16(darks))
    rec32.add_raw_projections(idx, raw_dev)
    reps = max(args.steps, 5)

    from tomography_local_demo_b200.recon import KernelTimer

    def timed(fn, rec):
        """Back-projection time per call: the device time of the call's launches (CUDA
        events right around each launch), so that the host's issue time between calls does
        not enter the comparison of the kernels."""
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        rec.kernel_timer = KernelTimer()
        for _ in range(reps):
            fn()
        kern = rec.kernel_timer.summary()
        rec.kernel_timer = None
        return sum(t for _, t in kern.values()) / 1e3 / reps

    t32 = timed(lambda: [rec32.reconstruct_planes_tensor([r]) for r in reqs], rec32)
    rec_bf16.reset()
    rec_bf16.add_raw_projections(idx, raw_dev)
    tbf = timed(lambda: rec_bf16.reconstruct_planes_tensor(reqs), rec_bf16)
    t32b = timed(lambda: rec32.reconstruct_planes_tensor(reqs), rec32)
    # the plain FP32 GPU path: direct global gathers (mr_backproject), one request per launch
    rec32.bp_kernel = "plain"
    t32p = timed(lambda: [rec32.reconstruct_planes_tensor([r]) for r in reqs], rec32)
    rec32.bp_kernel = "staged"
    # per-request latency of the 3-slice batch through the public API (host wall clock,
    # includes descriptor upload and the D2H of the images)
    lat = []
    for i in range(50 + 5):
        t0 = time.perf_counter()
        rec_bf16.reconstruct_planes(reqs)
        if i >= 5:
            lat.append((time.perf_counter() - t0) * 1e3)
    imgs = {f"bf16_store_{rec_bf16.filter_method}_filter": [x.cpu().numpy() for x in rec_bf16.reconstruct_planes_tensor(reqs)],
            "fp32_store_fft_filter": [x.cpu().numpy() for x in rec32.reconstruct_planes_tensor(reqs)]}
    return {
        "bp_only": {"bf16_batched_updates_per_s": updates / tbf,
                    "fp32_batched_updates_per_s": updates / t32b,
                    "fp32_one_request_per_launch_updates_per_s": updates / t32,
                    "fp32_plain_one_request_per_launch_updates_per_s": updates / t32p,
                    "bf16_batched_vs_fp32_per_request": t32 / tbf,
                    "bf16_batched_vs_plain_fp32_per_request": t32p / tbf},
        "latency_ms_3x512_batch": {"p50": float(np.percentile(lat, 50)),
                                   "p99": float(np.percentile(lat, 99)), "samples": len(lat)},
        "_images": imgs,
    }


def serving_simulation(args, dev, geom, raw_dev, flats, darks, store="bf16", max_batch=128):
    """Live-scan serving: the scan's raw views stream into the ring at 200 views/s (groups
    of 10) while slice requests arrive as a Poisson process at 500 req/s (sizes uniform in
    {128, 256, 512, 1024}^2, zoom 1-8, random orientation, COR offsets within +/-10 px),
    plus a 128^3 preview every 50 views; a SliceServer (20 GB admission budget) answers
    them: continuously batched on a BF16 ring by default, or one request per launch
    (max_batch=1) on an FP32 ring for the comparison. The request stream is the same
    seeded sequence for both. Reports p50/p99 submit-to-host latency and updates/s."""
    import torch
    from tomography_local_demo_b200 import SliceReconstructor
    from tomography_local_demo_b200.server import SliceServer
    from tomography_local_demo_b200.stream import AcquisitionSchedule
    rec = SliceReconstructor(None, geom, store=store, verbose=False, device=dev, filter=args.filter)
    rec.set_flat_dark(as_u16(flats), as_u16(darks))
    srv = SliceServer(rec, budget_bytes=20e9, max_batch=max_batch, pool_bytes=1 << 30)
    rng = np.random.default_rng(5)
    V, rate, req_rate = WORKLOAD["views"], 200.0, 500.0
    sched = AcquisitionSchedule(V, "interleaved", group=10, rate=rate)
    futs, previews = [], []
    # warm the server (first launches of each request kind: tile plans, module loading)
    first = sched.groups[0]
    rec.add_raw_projections(first, raw_dev[torch.from_numpy(first).to(dev)])
    for f in [srv.submit((0, 0, 0), (0, 0, 1), n=n) for n in (128, 1024)] + [srv.submit_preview(128)]:
        f.result()
    rec.reset()
    srv.latencies.clear()
    srv.latency_kinds.clear()
    srv.updates = 0
    # as in the other timed regions, no cyclic garbage collection while the scan runs: a
    # full collection pauses every thread of the process, the server's included
    gc.collect()
    gc.disable()
    t0 = time.perf_counter()
    next_req = t0 + rng.exponential(1.0 / req_rate)
    pushed, sent = 0, 0                 # groups and views pushed so far
    while pushed < len(sched):
        due = sched.due_by(time.perf_counter() - t0)
        if due > pushed:
            idx = np.concatenate(sched.groups[pushed:due])
            rec.add_raw_projections(idx, raw_dev[torch.from_numpy(idx).to(dev)])
            before, sent, pushed = sent, sent + len(idx), due
            if sent // 50 > before // 50:
                previews.append(srv.submit_preview(128))
        while next_req <= time.perf_counter():
            nrm = rng.normal(size=3)
            futs.append(srv.submit(tuple(rng.uniform(-10, 10) * nrm / np.linalg.norm(nrm)), tuple(nrm),
                                   n=int(rng.choice([128, 256, 512, 1024])), zoom=float(rng.uniform(1, 8)),
                                   cor_shift=float(rng.uniform(-10, 10))))
            next_req += rng.exponential(1.0 / req_rate)
        time.sleep(0.0005)
    for f in futs + previews:
        f.result()
    wall = time.perf_counter() - t0
    gc.enable()
    srv.device_status()
    srv.close()
    st = srv.stats()
    return {"requests": len(futs), "previews": len(previews), "batches": st["batches"],
            "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "slice_p50_ms": st["slice_p50_ms"],
            "slice_p99_ms": st["slice_p99_ms"], "wall_s": wall,
            "updates_per_s": st["updates"] / wall,
            "setup": "600 raw views at 200 views/s, Poisson 500 req/s, n in {128..1024}, zoom 1-8, "
                     f"COR +/-10 px, 128^3 preview per 50 views, {store} ring, "
                     + ("continuous batching" if max_batch > 1 else "one request per launch")
                     + ", 20 GB budget"}


def cpu_whole_job(raw, fl, dk, geom, reqs, box, reps, warmup=1, precision="ref"):
    """Time the whole job on the host with the oracle port: correction + FDK filter of all
    views, then every in-box pixel of every slice back-projected from all views. Returns
    (per-run job seconds, timings of the last run, values of the last run)."""
    for _ in range(warmup):
        cpu_job(raw, fl, dk, geom, reqs, box, precision)
    runs, tm, vals = [], None, None
    for _ in range(reps):
        t0 = time.perf_counter()
        vals, tm = cpu_job(raw, fl, dk, geom, reqs, box, precision)
        runs.append(time.perf_counter() - t0)
    return runs, tm, vals


def cpu_baseline_and_accuracy(args, geom, raw_dev, flats, darks, reqs, box, updates, imgs):
    raw = as_u16(raw_dev)
    fl, dk = as_u16(flats), as_u16(darks)
    V = WORKLOAD["views"]
    runs, tm, _ = cpu_whole_job(raw, fl, dk, geom, reqs, box, reps=3)
    t_job = float(np.median(runs))
    base = {"value": updates / t_job, "unit": "updates/s", "cores": tm["threads"], "kind": "port",
            "sample": (f"the whole job, measured (median of {len(runs)} runs after 1 warm-up): oracle port "
                       f"(C back-projection with FP64 accumulation, NumPy FDK filter) on {tm['threads']} host "
                       f"threads, correction + filter of all {V} views ({tm['t_filter']:.2f} s) and every "
                       f"in-box pixel of the 3 slices x {V} views ({tm['t_bp']:.2f} s); job "
                       f"{t_job:.2f} s (runs {', '.join(f'{r:.2f}' for r in runs)} s)")}
    acc = {}
    if imgs is not None:
        vals64, _ = cpu_job(raw, fl, dk, geom, reqs, box, "fp64")
        for store, ims in imgs.items():
            rl, mx = [], []
            for (sel, v64), im in zip(vals64, ims):
                got = im[sel].astype(np.float64)
                rl.append(float(np.linalg.norm(got - v64) / np.linalg.norm(v64)))
                mx.append(float(np.max(np.abs(got - v64))))
            acc[store] = {"rel_l2_vs_fp64": rl, "max_abs_err": mx}
        acc["sample"] = "every in-box pixel of each slice"
    return base, acc


# ------------------------------------------------------------------ reference arm
def run_reference(args, rank, world, local):
    """The reference's CPU implementation of the path (oracle port, all host threads) on
    the same workload: every step is the whole job, measured; the line reports the
    median step."""
    if rank != 0:
        return None
    import torch
    dev = torch.device("cuda", local) if torch.cuda.is_available() else torch.device("cpu")
    geom, raw_dev, flats, darks = make_scan(dev)
    raw, fl, dk = as_u16(raw_dev), as_u16(flats), as_u16(darks)
    box = geom.volume_box()
    reqs = slice_requests(box)
    V = WORKLOAD["views"]
    updates = sum(in_box_pixels(box, reqs)) * V
    t0 = time.perf_counter()
    runs, tm, _ = cpu_whole_job(raw, fl, dk, geom, reqs, box, reps=args.steps, warmup=args.warmup)
    wall = time.perf_counter() - t0
    t_job = float(np.median(runs))
    value = updates / t_job
    sample = (f"every step the whole job: correction + FDK filter of all {V} views and every in-box pixel "
              f"of the 3 slices back-projected from {V} views (C port of the Numba kernel, FP64 "
              f"accumulation), on {tm['threads']} host threads; median of {len(runs)} steps "
              f"(min {min(runs):.3f} s, max {max(runs):.3f} s)")
    return {"metric": "voxel-proj updates/s", "value": value, "unit": "updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_job * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD_NAME, "views": V, "rows": WORKLOAD["rows"],
                       "cols": WORKLOAD["cols"], "slices": len(reqs), "n": WORKLOAD["n"],
                       "store": "fp32", "accumulate": "f64", "parallelism": "host threads"},
            "cpu_baseline": {"value": value, "unit": "updates/s", "cores": tm["threads"],
                             "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "timing": {"filter_s_last": tm["t_filter"], "bp_s_last": tm["t_bp"],
                       "step_s": [round(r, 4) for r in runs]},
            "wall_s": wall}


# ------------------------------------------------------------------ single-kernel cases
def run_case(args):
    """One kernel family on its own, device-timed with CUDA events (no host copies):
    otsu        the three voxel passes of model.otsu_threshold on a 640^3 float32 volume
    surface     model.marching_cubes of a 640^3 float32 volume (a noisy ball of radius 250)
    correct     the loaders' correction + crop (mr_correct_u16) of 120 views 1944 x 1536
    ingest-full the fused FFT ingest of 1200 raw views 1944 x 1536 into a bf16 ring
    parker      the ingest of a 600-view short scan (pi + fan angle) of 486 x 384 raw views
                with Parker weights (correction, weighting, tensor-core filter), beside
                the same ingest without them
    wire        a scan through the wire-compatible service on 127.0.0.1: per step, reset,
                600 raw views of 486 x 384 pushed in messages of 50 views, then three
                512^2 slices back in one BF16 reply (host wall clock)
    Prints one JSON line: the case's own throughput and its HBM figure."""
    import torch
    from tomography_local_demo_b200 import SliceReconstructor, circular_cone_vectors
    from tomography_local_demo_b200 import _native as N
    from tomography_local_demo_b200.model import otsu_threshold
    dev = torch.device("cuda", 0)
    gen = torch.Generator(device=dev)
    gen.manual_seed(1)
    if args.case == "otsu":
        vol = torch.rand((640, 640, 640), generator=gen, device=dev) * 0.5
        vol[vol < 0.05] = 0
        step = lambda: otsu_threshold(vol)                        # noqa: E731 (waits for its result)
        units, unit, nbytes = vol.numel(), "voxels/s", 5 * vol.numel() * 4     # 5 passes over the voxels
    elif args.case == "surface":
        from tomography_local_demo_b200.model import marching_cubes
        x = torch.arange(640, device=dev, dtype=torch.float32) - 319.5
        vol = 250.0 - torch.sqrt(x[:, None, None] ** 2 + x[None, :, None] ** 2 + x[None, None, :] ** 2)
        vol += 0.3 * torch.randn(vol.shape, generator=gen, device=dev)
        step = lambda: marching_cubes(vol, 0.0, (0.0, 0.0, 0.0), 0.0825)   # noqa: E731
        units, unit, nbytes = vol.numel(), "voxels/s", 2 * vol.numel() * 4     # two passes over the voxels
    elif args.case == "correct":
        k, R0, C0 = args.case_views or 120, 1536, 1944
        raw = torch.randint(30000, 50000, (k, R0, C0), generator=gen, device=dev, dtype=torch.int32).to(torch.int16)
        dark = torch.full((R0, C0), 100.0, device=dev)
        gain = torch.full((R0, C0), 1.0 / 49900.0, device=dev)
        out = torch.empty((R0, k, C0), device=dev)
        lib, v = N.load(), ctypes.c_void_p

        def step():
            N.check(lib.mr_correct_u16(v(raw.data_ptr()), R0 * C0, C0, k, 1, 1, R0, 0, 0, R0, C0, v(dark.data_ptr()),
                                       v(gain.data_ptr()), C0, N.MR_CORRECT_FLEXRAY, v(out.data_ptr()), k * C0, C0,
                                       v(torch.cuda.current_stream().cuda_stream)), "mr_correct_u16")
        units, unit, nbytes = k, "views/s", k * R0 * C0 * (2 + 4)
    elif args.case == "parker":
        V, R0, C0 = args.case_views or 600, 384, 486
        w = WORKLOAD
        fan = float(np.arctan(0.5 * C0 * w["pixel"] / w["sdd"]))
        # the last view sits one step short of the range: cover 180 deg + fan angle with it
        geom = circular_cone_vectors(V, w["sod"], w["sdd"], R0, C0, w["pixel"],
                                     angular_range=(np.pi + 2 * fan) * V / (V - 1) * 1.001)
        raw = torch.randint(30000, 50000, (V, R0, C0), generator=gen, device=dev, dtype=torch.int32).to(torch.int16)
        recs = {}
        for pk in (True, False):
            recs[pk] = SliceReconstructor(None, geom, store="bf16", verbose=False, filter="tc", parker=pk)
            recs[pk].set_flat_dark(np.full((2, R0, C0), 50000, np.uint16), np.full((2, R0, C0), 100, np.uint16))
        idx = np.arange(V)

        def ingest(rec):
            rec.reset()
            rec.add_raw_projections(idx, raw)
            torch.cuda.current_stream().wait_stream(rec.ingest_stream)
        step = lambda: ingest(recs[True])                          # noqa: E731
        units, unit, nbytes = V, "views/s", V * R0 * C0 * (2 + 2)
        for _ in range(args.warmup):
            ingest(recs[False])
        torch.cuda.synchronize()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record()
        for _ in range(args.steps):
            ingest(recs[False])
        a1.record()
        torch.cuda.synchronize()
        extra = {"without_parker_ms": a0.elapsed_time(a1) / args.steps}
    elif args.case == "wire":
        return run_wire_case(args)
    else:
        V, R0, C0 = args.case_views or 1200, 1536, 1944
        geom = circular_cone_vectors(V, 440.0, 680.0, R0, C0, 0.0748)
        raw = torch.randint(30000, 50000, (V, R0, C0), generator=gen, device=dev, dtype=torch.int32).to(torch.int16)
        rec = SliceReconstructor(None, geom, window="ram-lak", store="bf16", verbose=False, filter="fft")
        rec.set_flat_dark(np.full((2, R0, C0), 50000, np.uint16), np.full((2, R0, C0), 100, np.uint16))
        idx = np.arange(V)

        def step():
            rec.reset()
            rec.add_raw_projections(idx, raw)
            torch.cuda.current_stream().wait_stream(rec.ingest_stream)   # the timed stream sees it
        units, unit, nbytes = V, "views/s", V * R0 * C0 * (2 + 2)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak, source = float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError):
        peak, source = 6650.0, "fallback"
    gbs = nbytes / ms / 1e6
    line = {"case": args.case, "metric": unit.split("/")[0] + " per second", "value": units / ms * 1e3,
            "unit": unit, "ms_per_step": ms, "steps": args.steps, "warmup": args.warmup,
            "hbm": {"algorithmic_bytes": nbytes, "achieved_gbs": gbs, "peak_gbs": peak, "frac": gbs / peak,
                    "peak_source": source}}
    if args.case == "parker":
        line.update(extra)
    return line


def _events_ms(fn, stream, steps, warmup):
    """Average device time (ms) of fn() over `steps` calls after `warmup`, CUDA events on
    the stream fn launches on."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        fn()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / steps


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _issue_roofline(updates, ms, ops_per_update=FP32_LANE_OPS_PER_UPDATE):
    ach = updates * ops_per_update / (ms / 1e3) / 1e12
    peak = NOMINAL_FP32_LANE_OPS / 1e12
    return {"bound": "fp32-issue", "achieved": ach, "peak": peak, "unit": "T FP32-lane-ops/s",
            "frac": ach / peak, "ops_per_update": ops_per_update, "updates_per_s": updates / (ms / 1e3),
            "peak_source": "nominal (148 SMs x 128 FP32 lanes x 1965 MHz); not in MEASURED_PEAKS.json"}


def _hbm_roofline(nbytes, ms):
    pk = _peaks()
    peak = float(pk.get("hbm_gbs", 6650.0))
    ach = nbytes / (ms / 1e3) / 1e9
    return {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
            "algorithmic_bytes": nbytes, "peak_source": "measured" if "hbm_gbs" in pk else "fallback"}


KERNEL_CASES = ("bp-plain", "bp-persistent", "grad", "entropy", "preprocess")


def run_kernel_case(args):
    """Kernels outside the headline step, each on the bench scan (600 raw views of
    486 x 384 ingested into a ring), device-timed with CUDA events:
    bp-plain       mr_backproject (direct global gathers, FP32 ring), the 3 bench slices in one launch
    bp-persistent  mr_backproject_persistent (the launch the slice server replays), BF16 ring,
                   the 3 bench slices, tiles pulled from a device work counter
    grad           the differentiable back-projector on the FP32 ring over the calibration's two
                   192^2 slices (axial at z = 0, central x-z) at COR +1.7 px, tilt 0.3 deg:
                   mr_backproject_matched, mr_project_adjoint (the matched forward projector),
                   mr_bp_grad_geom (d/dCOR, d/dtilt); each warm-up round launches each once
    entropy        mr_slice_entropy of the 25 trial 192^2 slices of estimate_cor
    preprocess     tilt rotation (0.3 deg) then Gaussian (sigma 1 px) of the 600-view block
                   [384, 600, 486] f32 (mr_rotate_f32, mr_gaussian_axis_f32 x 2); each warm-up
                   round launches the rotation, then the two Gaussian passes"""
    import torch
    from tomography_local_demo_b200 import SliceReconstructor
    from tomography_local_demo_b200 import _native as N
    from tomography_local_demo_b200 import preprocess as PP
    from tomography_local_demo_b200.recon import ctypes_void as cv
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    geom, raw_dev, flats, darks = make_scan(dev)
    box = geom.volume_box()
    reqs = slice_requests(box)
    V = WORKLOAD["views"]
    idx = np.arange(V)
    store = {"bp-plain": "fp32", "grad": "fp32"}.get(args.case, "bf16")
    rec = SliceReconstructor(None, geom, store=store, verbose=False, device=dev, filter="fft")
    rec.set_flat_dark(as_u16(flats), as_u16(darks))
    rec.add_raw_projections(idx, raw_dev)
    torch.cuda.synchronize()
    steps, warm = args.steps, args.warmup
    line = {"case": args.case, "steps": steps, "warmup": warm}
    lib = N.load()
    if args.case in ("bp-plain", "bp-persistent"):
        updates = sum(in_box_pixels(box, reqs)) * V
        if args.case == "bp-plain":
            rec.bp_kernel = "plain"
            ms = _events_ms(lambda: rec.reconstruct_planes_tensor(reqs), rec.stream, steps, warm)
            name = "mr_backproject"
        else:
            grids = np.zeros(len(reqs), dtype=N.GRID_DTYPE)
            off = 0
            for r, q in enumerate(reqs):
                grids[r] = rec.plane_grid(q["origin"], q["normal"], q["n"])
                grids[r]["out_offset"] = off
                off += q["n"] ** 2
            grids["n_views"], grids["scale"] = V, np.pi / V
            tiles = N.plan_tiles(grids, rec._band_axis)
            recs = torch.from_numpy(np.concatenate([grids.view(np.uint8), tiles.view(np.uint8)])).to(dev)
            nt = torch.tensor([len(tiles)], dtype=torch.int64, device=dev)
            counter = torch.zeros(1, dtype=torch.int32, device=dev)
            status = torch.zeros(1, dtype=torch.int32, device=dev)
            out = torch.empty(off, dtype=torch.float32, device=dev)
            st = torch.cuda.current_stream(dev)

            def launch():
                N.check(lib.mr_backproject_persistent(
                    rec._ring_c, cv(rec._views_dev.data_ptr()), cv(recs.data_ptr()),
                    cv(recs.data_ptr() + grids.nbytes), cv(nt.data_ptr()), len(tiles), cv(counter.data_ptr()),
                    cv(out.data_ptr()), cv(status.data_ptr()), cv(st.cuda_stream)), "mr_backproject_persistent")
            ms = _events_ms(launch, st, steps, warm)
            assert int(status.item()) == 0, "a bounded device-side wait gave up"
            name = "mr_backproject_persistent"
        line.update(kernel=name, workload="3 oblique 512^2 slices x 600 views, " + store + " ring",
                    ms=ms, updates=updates, roofline=_issue_roofline(updates, ms))
    elif args.case == "grad":
        creqs = [dict(origin=(0.0, 0.0, 0.0), normal=(0.0, 0.0, 1.0), n=192),
                 dict(origin=(0.0, 0.0, 0.0), normal=(0.0, 1.0, 0.0), n=192)]
        op = rec.bp_operator(creqs)
        q = rec._ring
        shift, tilt = 1.7, float(np.deg2rad(0.3))
        st = torch.cuda.current_stream(dev)
        f = op.forward(q, shift, tilt)
        updates = int((f != 0).sum()) * V
        y = torch.randn(op.n_out, generator=torch.Generator(device=dev).manual_seed(3), device=dev)
        fns = [lambda: op.forward(q, shift, tilt), lambda: op.adjoint(y, shift, tilt, tuple(q.shape)),
               lambda: op.grad_geometry(q, y, shift, tilt)]
        for _ in range(warm):              # one launch of each kernel per warm-up round
            for fn in fns:
                fn()
        ms_f, ms_a, ms_g = (_events_ms(fn, st, steps, 0) for fn in fns)
        line.update(workload="2 calibration slices 192^2 (axial z=0, x-z) x 600 views, fp32 ring, "
                             "COR +1.7 px, tilt 0.3 deg", updates=updates,
                    kernels={"mr_backproject_matched": {"ms": ms_f, "roofline": _issue_roofline(updates, ms_f)},
                             "mr_project_adjoint": {"ms": ms_a, "roofline": _issue_roofline(updates, ms_a),
                                                    "atomics_per_s": 4 * updates / (ms_a / 1e3),
                                                    "note": "time includes zeroing the 448 MB gradient ring"},
                             "mr_bp_grad_geom": {"ms": ms_g, "roofline": _issue_roofline(updates, ms_g)}})
    elif args.case == "entropy":
        shifts = np.arange(-3.0, 3.01, 0.25)
        creqs = [dict(origin=(0.0, 0.0, 0.0), normal=(0.0, 0.0, 1.0), n=192, cor_shift=float(s)) for s in shifts]
        imgs, _ = rec._planes(creqs)
        torch.cuda.synchronize()
        scores = torch.empty(len(creqs), dtype=torch.float64, device=dev)
        st = torch.cuda.current_stream(dev)
        n2 = 192 * 192

        def launch():
            N.check(lib.mr_slice_entropy(cv(imgs.data_ptr()), len(creqs), n2, n2, 128, cv(scores.data_ptr()),
                                         cv(st.cuda_stream)), "mr_slice_entropy")
        ms = _events_ms(launch, st, steps, warm)
        nbytes = 2 * len(creqs) * n2 * 4           # two passes over the pixels (range, then bins)
        line.update(kernel="mr_slice_entropy", workload="25 trial axial slices 192^2, 128 bins", ms=ms,
                    roofline=_hbm_roofline(nbytes, ms),
                    note="one CTA per trial slice: 25 CTAs on 148 SMs, 3.7 MB that stays in L2")
    elif args.case == "preprocess":
        R, C = WORKLOAD["rows"], WORKLOAD["cols"]
        x = torch.rand((R, V, C), generator=torch.Generator(device=dev).manual_seed(1), device=dev)
        st = torch.cuda.current_stream(dev)
        fns = [lambda: PP._rotate_dev(x, -0.3), lambda: PP._gaussian_dev(x, 1.0)]
        for _ in range(warm):              # rotation, then the two Gaussian passes, per round
            for fn in fns:
                fn()
        ms_r, ms_g = (_events_ms(fn, st, steps, 0) for fn in fns)
        px = R * V * C
        line.update(workload="block [384, 600, 486] f32 (448 MB)",
                    kernels={"mr_rotate_f32": {"ms": ms_r, "roofline": _hbm_roofline(8 * px, ms_r)},
                             "mr_gaussian_axis_f32 (rows, then cols)": {"ms": ms_g,
                                                                        "roofline": _hbm_roofline(16 * px, ms_g)}})
    return line


def run_wire_case(args):
    """The `wire` case of run_case: host wall clock per step through net.Server."""
    import threading
    import torch
    from tomography_local_demo_b200 import net
    dev = torch.device("cuda", 0)
    geom, raw_dev, flats, darks = make_scan(dev)
    raw = raw_dev.cpu().numpy().view(np.uint16)
    reqs = slice_requests(geom.volume_box())
    srv = net.Server(port=0, verbose=False, store="bf16", filter="tc", budget_bytes=1 << 30)
    address = srv.listen()
    threading.Thread(target=srv.serve_forever, daemon=True).start()
    sink = net.RemoteSink(address, geom)
    sink.set_flat_dark(as_u16(flats), as_u16(darks))
    view = net.RemoteReconstructor(address, encoding="bf16")
    V, group = WORKLOAD["views"], 50

    def step():
        sink.reset()
        for g0 in range(0, V, group):
            idx = np.arange(g0, min(V, g0 + group))
            sink.add_raw_projections(idx, raw[idx])
        return view.reconstruct_planes(reqs)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    ms = (time.perf_counter() - t0) / args.steps * 1e3
    for c in (view, sink):
        c.close()
    srv.close()
    raw_bytes = raw.nbytes
    reply = sum(r["n"] ** 2 for r in reqs) * 2
    return {"case": "wire", "metric": "views per second", "value": V / ms * 1e3, "unit": "views/s",
            "ms_per_step": ms, "steps": args.steps, "warmup": args.warmup, "clock": "host wall clock",
            "bytes_per_step": {"requests": raw_bytes, "replies": reply},
            "wire_gbs": (raw_bytes + reply) / ms / 1e6}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--store", choices=("fp32", "bf16", "fp16"), default="bf16")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline / accuracy leg")
    ap.add_argument("--no-serve", action="store_true", help="skip the live-scan serving simulation")
    ap.add_argument("--filter", choices=("fft", "tc", "tc-bf16"), default="tc",
                    help="row filter: shared-memory FFT or tensor-core Toeplitz GEMM (split FP16 / BF16)")
    ap.add_argument("--case", choices=("otsu", "surface", "correct", "ingest-full", "parker", "wire") + KERNEL_CASES,
                    default=None,
                    help="time one other kernel family alone instead of the headline step")
    ap.add_argument("--case-views", type=int, default=0, help="views of the correct / ingest-full case")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.case in KERNEL_CASES:
        print(json.dumps(run_kernel_case(args)), flush=True)
        return
    if args.case is not None:
        print(json.dumps(run_case(args)), flush=True)
        return
    rank, world, local = dist_setup()
    try:
        line = (run_reference if args.impl == "reference" else run_ours)(args, rank, world, local)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
