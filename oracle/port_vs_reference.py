"""TEST INFRASTRUCTURE ONLY. Times the oracle port (the CPU baseline of the bench) against
the reference's own CPU implementation on the same host, thread count and workload, to
show that the port is representative of the reference's speed.

    python oracle/port_vs_reference.py PATH-TO-REFERENCE-CHECKOUT [--threads N] [--reps 3]

Workload: the bench scan (600 cone views of 486 x 384, 40 seeded ellipsoids; line
integrals without noise, since only the timing matters) and its three oblique 512^2
slices. Compared, median of `reps` runs each:
  filter : minirecast SliceReconstructor(proj, geom, backend="numba") construction, which
           filters all views in 64-view chunks (recon.py:298-343, 85-104), against the
           port's FDK filter (oracle/filter.py) on the same views;
  bp     : SliceReconstructor.reconstruct_plane of the three slices after warmup()
           (recon.py:426-440 -> bp_cone_numba, recon.py:193-219), against the port's C
           back-projection (oracle/bp_oracle.c) of the same in-box points.
Prints one JSON line. The reference runs from a copy (Numba's cache writes next to it).
"""
import argparse
import json
import os
import shutil
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("reference")
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args()
    os.environ["NUMBA_NUM_THREADS"] = str(a.threads)
    tmp = tempfile.mkdtemp(prefix="minirecast_ref_")
    shutil.copytree(os.path.join(a.reference, "minirecast"), os.path.join(tmp, "minirecast"))
    sys.path.insert(0, tmp)
    import numba
    from minirecast import geometry as RG
    from minirecast import recon as RR

    import bench
    from oracle import bp as obp
    from oracle import filter as of
    from oracle import geometry as og
    from tomography_local_demo_b200 import phantom as PH

    w = bench.WORKLOAD
    geom = bench.geometry()
    ph = PH.EllipsoidPhantom(1.0, PH.random_ellipsoids(w["ellipsoids"], w["phantom_seed"]))
    lines = PH.project_cone_torch(ph, geom, device="cpu").numpy()          # [A, R, C]
    proj = np.ascontiguousarray(np.transpose(lines, (1, 0, 2)))             # [R, A, C]
    rgeom = RG.circular_cone_vectors(w["views"], w["sod"], w["sdd"], w["rows"], w["cols"], w["pixel"])
    box = rgeom.volume_box()
    reqs = bench.slice_requests(box)
    numba.set_num_threads(a.threads)
    obp.build()
    obp.threads(a.threads)

    def med(fn):
        ts = []
        for _ in range(a.reps):
            t0 = time.perf_counter()
            fn()
            ts.append(time.perf_counter() - t0)
        return float(np.median(ts)), ts

    # ---- filter
    holder = {}

    def ref_filter():
        holder["rec"] = RR.SliceReconstructor(proj, rgeom, window="shepp-logan", backend="numba", verbose=False)
    t_ref_f, ts_ref_f = med(ref_filter)
    rec = holder["rec"]
    K = of.cone_constants(geom.vectors)
    from concurrent.futures import ThreadPoolExecutor
    A = w["views"]
    q = np.zeros((A, w["rows"], w["cols"]), np.float32)

    def port_filter():
        def chunk(i0):
            i1 = min(A, i0 + 16)
            Kc = {k: v[i0:i1] for k, v in K.items()}
            return i0, of.fdk_filter_block(proj[:, i0:i1], Kc, "shepp-logan")
        with ThreadPoolExecutor(a.threads) as ex:
            for i0, part in ex.map(chunk, range(0, A, 16)):
                q[i0:i0 + len(part)] = part
    t_port_f, ts_port_f = med(port_filter)
    filt_diff = float(np.abs(q - rec._q[:A]).max() / np.abs(rec._q[:A]).max())

    # ---- back-projection of the three slices
    rec.warmup()
    pts_all = [og.slice_points(box, r["origin"], r["normal"], r["n"]) for r in reqs]
    updates = sum(int(m.sum()) for _, m in pts_all) * A

    def ref_bp():
        for r in reqs:
            rec.reconstruct_plane(r["origin"], r["normal"], n=r["n"])
    t_ref_b, ts_ref_b = med(ref_bp)

    def port_bp():
        for pts, m in pts_all:
            obp.bp_cone(q, K["s"], K["d"], K["uu"], K["vv"], K["n"], K["sdd"], K["sod"], pts[m], np.pi / A)
    t_port_b, ts_port_b = med(port_bp)
    img_ref, _ = rec.reconstruct_plane(reqs[0]["origin"], reqs[0]["normal"], n=reqs[0]["n"])
    pts, m = pts_all[0]
    v = obp.bp_cone(q, K["s"], K["d"], K["uu"], K["vv"], K["n"], K["sdd"], K["sod"], pts[m], np.pi / A)
    bp_diff = float(np.linalg.norm(v - img_ref[m]) / np.linalg.norm(img_ref[m]))
    print(json.dumps({
        "threads": a.threads, "reps": a.reps, "views": A, "updates": updates,
        "filter_s": {"reference_numba_constructor": t_ref_f, "port": t_port_f, "ratio_ref_over_port": t_ref_f / t_port_f,
                     "runs_ref": ts_ref_f, "runs_port": ts_port_f, "max_rel_diff": filt_diff},
        "bp_s": {"reference_reconstruct_plane_x3": t_ref_b, "port": t_port_b, "ratio_ref_over_port": t_ref_b / t_port_b,
                 "reference_updates_per_s": updates / t_ref_b, "port_updates_per_s": updates / t_port_b,
                 "runs_ref": ts_ref_b, "runs_port": ts_port_b, "rel_l2_slice0": bp_diff},
        "job_s": {"reference": t_ref_f + t_ref_b, "port": t_port_f + t_port_b},
    }))


if __name__ == "__main__":
    main()
