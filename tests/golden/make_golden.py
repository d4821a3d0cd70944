"""Generate the golden fixtures of tests/golden/ by running the REFERENCE itself.

    python tests/golden/make_golden.py PATH-TO-REFERENCE-CHECKOUT [--net-only]
    MINIRECAST_REF=PATH-TO-REFERENCE-CHECKOUT python tests/golden/make_golden.py

Imports minirecast (ZYHuang216/Tomography-local-demo) from the checkout given as the
argument or in the MINIRECAST_REF environment variable (one of them is required), runs its own functions on small seeded inputs and writes
compressed .npz fixtures next to this script. The tests only read the .npz files; the
reference is not needed to run them. Numba's cache goes to a temporary directory so a
read-only checkout works.
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root):
    os.environ.setdefault("NUMBA_CACHE_DIR", tempfile.mkdtemp(prefix="numba_cache_"))
    sys.path.insert(0, ref_root)
    import minirecast
    from minirecast import recon as R, preprocess as P, phantom as PH, geometry as G
    from minirecast import stream as S, model as M, hdf5 as H5, flexray as FX

    rng = np.random.default_rng(20240607)
    save = lambda name, **kw: np.savez_compressed(os.path.join(HERE, name), **kw)  # noqa: E731

    # ---------------------------------------------------------- ramp_response
    d = {}
    for n in (20, 128, 486):
        for tau in (1.0, 0.19245):
            for w in ("ram-lak", "shepp-logan", "hann", "cosine"):
                H, N = R.ramp_response(n, tau, w)
                d[f"H_{n}_{tau}_{w}"] = H
    save("ramp.npz", **d)

    # ---------------------------------------------------------- filter_rows
    x = rng.normal(0.0, 1.0, (3, 4, 50)).astype(np.float32)
    d = {"x": x}
    for w in ("ram-lak", "shepp-logan", "hann", "cosine"):
        d[f"y_{w}"] = R.filter_rows(x, 0.9, w)
    d["y64_shepp-logan"] = R.filter_rows(x.astype(np.float64), 0.9, "shepp-logan")
    save("filter_rows.npz", **d)

    # ---------------------------------------------------------- cone constants / FDK block
    geo = G.circular_cone_vectors(7, 300.0, 600.0, 16, 20, 1.5, det_shift_u=2.0)
    V = geo.vectors.copy()
    V_gen = V + rng.normal(0.0, 0.05, V.shape)          # generic (non-ideal) vectors
    K = R.cone_constants(V_gen)
    block = rng.normal(0.5, 0.2, (16, 7, 20)).astype(np.float32)
    d = {"V_ideal": V, "V_gen": V_gen, "block": block}
    for k, v in K.items():
        d["K_" + k] = v
    d["fdk_shepp-logan"] = R.fdk_filter_block(block, K, "shepp-logan")
    d["fdk_ram-lak"] = R.fdk_filter_block(block, K, "ram-lak")
    d["par_hann"] = np.transpose(R.filter_rows(block, 0.8, "hann"), (1, 0, 2))
    save("fdk.npz", **d)

    # ---------------------------------------------------------- back-projection kernels
    A, Rr, Cc = 12, 16, 20
    q = rng.normal(0.0, 1.0, (A, Rr, Cc)).astype(np.float32)
    geo = G.circular_cone_vectors(A, 60.0, 100.0, Rr, Cc, 1.0)
    Vb = geo.vectors + rng.normal(0.0, 0.02, geo.vectors.shape)
    Kb = R.cone_constants(Vb)
    pts = rng.uniform(-14.0, 14.0, (300, 3))
    shift = 0.7
    Dshift = Kb["d"] - shift * Kb["u"]
    args = (q, Kb["s"], Dshift, Kb["uu"], Kb["vv"], Kb["n"], Kb["sdd"], Kb["sod"], pts, np.pi / A)
    d = {"q": q, "V": Vb, "pts": pts, "shift": shift,
         "cone_numba": R.bp_cone_numba(*args), "cone_numpy": R.bp_cone_numpy(*args)}
    ang = np.arange(A) * np.pi / A + 0.01
    pargs = (q, np.cos(ang), np.sin(ang), 0.9, 1.1, pts, np.pi / A, -1.3)
    d.update(angles=ang, par_numba=R.bp_parallel_numba(*pargs), par_numpy=R.bp_parallel_numpy(*pargs))
    save("bp.npz", **d)

    # ---------------------------------------------------------- preprocess
    b = rng.normal(1.0, 0.3, (20, 3, 25)).astype(np.float32)
    img = np.zeros((41, 1, 41), np.float32)
    img[20, 0, 30] = 1.0
    save("preprocess.npz", block=b, gauss_1_5=P.gaussian_blur(b, 1.5), rot_7=P.rotate_projections(b, 7.0),
         apply=P.apply(b, gaussian=0.8, tilt=2.5), point=img, rot_90=P.rotate_projections(img, 90.0))

    # ---------------------------------------------------------- phantom
    ph = PH.EllipsoidPhantom(scale=50.0)
    ppts = rng.uniform(-50, 50, (200, 3))
    starts = rng.uniform(-60, 60, (50, 3))
    dirs = rng.normal(size=(50, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    pg = G.ParallelGeometry(np.arange(9) * np.pi / 9, 10, 12, 9.0, 11.0)
    cg = G.circular_cone_vectors(9, 300.0, 600.0, 10, 12, 15.0, det_shift_u=1.5)
    save("phantom.npz", pts=ppts, evaluate=ph.evaluate(ppts), starts=starts, dirs=dirs,
         lines=ph.line_integrals(starts, dirs), par=PH.project_parallel(ph, pg),
         cone=PH.project_cone(ph, cg), cone_V=cg.vectors)

    # ---------------------------------------------------------- end-to-end reconstructor
    for name in ("cone", "parallel"):
        if name == "cone":
            geom = G.circular_cone_vectors(40, 300.0, 600.0, 24, 32, 7.0, det_shift_u=1.0)
            proj = PH.project_cone(ph, geom)
            extra = {"V": geom.vectors}
        else:
            geom = G.ParallelGeometry(np.arange(36) * np.pi / 36, 20, 32, 3.5, 4.4)
            proj = PH.project_parallel(ph, geom)
            extra = {"angles": geom.angles}
        rec = R.SliceReconstructor(proj, geom, backend="numba", verbose=False)
        img1, _ = rec.reconstruct_plane((3.0, -2.0, 5.0), (1.0, 0.5, 0.8), n=40, size=110)
        img2, _ = rec.reconstruct_plane((0, 0, 1.0), (0.3, 0.0, 1.0), n=33, zoom=1.5,
                                        center=(2.0, 0, 0), cor_shift=0.8)
        img3, _ = rec.reconstruct_plane((0, 0, 0), (0, 0, 1), n=24)
        vol, origin, h = rec.reconstruct_volume(voxel=8.0)
        best, scores = rec.estimate_cor(np.arange(-2.0, 2.01, 0.5), n=32, verbose=False)
        live = R.SliceReconstructor(None, geom, backend="numba", verbose=False)
        order = S.arrival_order(geom.n_angles, "interleaved")
        for i in range(0, len(order), 7):
            idx = order[i:i + 7]
            live.add_projections(idx, proj[:, idx, :])
        img_live, _ = live.reconstruct_plane((0, 0, 1.0), (0.3, 0.0, 1.0), n=33, zoom=1.5,
                                             center=(2.0, 0, 0), cor_shift=0.8)
        save(f"recon_{name}.npz", proj=proj, rows=geom.rows, cols=geom.cols,
             box=rec.box, img_oblique=img1, img_zoom=img2, img_axial=img3, vol=vol,
             vol_origin=origin, vol_h=h, cor_best=best, cor_scores=scores,
             img_live=img_live, live_order=live._order[:live.n], **extra)

    # ---------------------------------------------------------- loaders (raw correction)
    pgeo = G.ParallelGeometry(np.arange(8) * np.pi / 8, 12, 16, 1.7, 1.7)
    p = PH.project_parallel(ph, pgeo) * 0.01
    flat, dark = 5000.0, 100.0
    data = (dark + (flat - dark) * np.exp(-p)).transpose(1, 0, 2)
    data = (data + rng.normal(0, 30, data.shape)).clip(0, 65535).astype(np.uint16)
    whites = (rng.normal(flat, 50, (2, 12, 16))).astype(np.uint16)
    darks = (rng.normal(dark, 3, (2, 12, 16))).astype(np.uint16)
    files = {"exchange/data": data, "exchange/data_white": whites, "exchange/data_dark": darks,
             "exchange/theta": np.rad2deg(pgeo.angles)}

    class F(dict):
        def __enter__(self):
            return self

        def __exit__(self, *a):
            return False

    class FakeH5:
        @staticmethod
        def File(path, mode):
            return F(files)

    proj_h5, _ = H5.load_dxchange("fake.h5", sample=2, h5=FakeH5, verbose=False)

    # FleX-ray: uint16 TIFFs written with PIL into a temporary scan folder
    from PIL import Image
    tmp = tempfile.mkdtemp(prefix="flexray_")
    R0, C0, nsc = 12, 18, 4
    raws = rng.integers(2000, 40000, (nsc, R0, C0)).astype(np.uint16)
    fl = rng.integers(45000, 52000, (2, R0, C0)).astype(np.uint16)
    dk = rng.integers(90, 110, (2, R0, C0)).astype(np.uint16)
    for i, im in enumerate(raws):
        Image.fromarray(im).save(os.path.join(tmp, f"scan_{i:06d}.tif"))
    for i, im in enumerate(fl):
        Image.fromarray(im).save(os.path.join(tmp, f"io{i:06d}.tif"))
    for i, im in enumerate(dk):
        Image.fromarray(im).save(os.path.join(tmp, f"di{i:06d}.tif"))
    with open(os.path.join(tmp, "scan settings.txt"), "w") as f:
        f.write("SOD: 300\nSDD: 600\nVoxel size: 100\nStart angle: 0\nLast angle: 360\n")
    proj_fx, _ = FX.load_flexray(tmp, sample=2, skip=1, profile="none", auto_box=False, crop=False,
                                 verbose=False)
    save("loaders.npz", h5_data=data, h5_white=whites, h5_dark=darks, h5_proj=proj_h5,
         fx_raw=raws, fx_flat=fl, fx_dark=dk, fx_proj=proj_fx)

    # ---------------------------------------------------------- stream order / Otsu
    d = {f"order_{n}": S.arrival_order(n, "interleaved") for n in (1, 2, 10, 17, 64, 600)}
    vol = rng.gamma(2.0, 0.1, (10, 11, 12)).astype(np.float32)
    vol[vol < 0.05] = 0
    save("misc.npz", otsu_vol=vol, otsu=M.otsu_threshold(vol), **d)
    loader_fixtures(FX, H5, save)
    net_fixtures(save)
    print("golden fixtures written to", HERE, "from minirecast", minirecast.__version__)


class _Recorder:
    """A connection stand-in that keeps every payload passed to send_bytes."""

    def __init__(self):
        self.payloads = []

    def send_bytes(self, b):
        self.payloads.append(bytes(b))


def net_messages():
    """(header, array) pairs covering the reference's message kinds."""
    rng = np.random.default_rng(11)
    return [({"cmd": "hello", "role": "adapter"}, None),
            ({"cmd": "projections", "indices": [3, 1, 2]}, rng.normal(size=(4, 3, 5)).astype(np.float32)),
            ({"version": 7}, rng.normal(size=(6, 6)).astype(np.float32)),
            ({"origin": [0.5, -1.0, 2.0], "spacing": 0.25}, rng.gamma(2.0, 1.0, (2, 3, 4)).astype(np.float32)),
            ({"cmd": "raw", "note": "u16"}, rng.integers(0, 65535, (2, 3, 4)).astype(np.uint16)),
            ({"cmd": "slice", "origin": [0.0, 0.0, 0.0], "normal": [0.0, 0.0, 1.0], "n": 64, "zoom": 1.0,
              "center": None}, None)]


def net_fixtures(save):
    """Payloads of the reference's net.send for the messages of net_messages(), and its
    geometry messages for a cone and a parallel scan."""
    from minirecast import net as NET, geometry as G
    out = {}
    for i, (h, arr) in enumerate(net_messages()):
        rec = _Recorder()
        NET.send(rec, h, arr)
        for j, b in enumerate(rec.payloads):
            out[f"m{i}_p{j}"] = np.frombuffer(b, dtype=np.uint8)
        out[f"m{i}_count"] = np.array(len(rec.payloads))
    cone = G.circular_cone_vectors(12, 300.0, 600.0, 8, 10, 1.5, det_shift_u=0.7)
    par = G.ParallelGeometry(np.linspace(0, np.pi, 9, endpoint=False), 6, 7, 0.5, 0.25)
    for tag, geom in (("cone", cone), ("par", par)):
        h, arr = NET.geometry_message(geom)
        rec = _Recorder()
        NET.send(rec, h, arr)
        out[f"geom_{tag}_p0"] = np.frombuffer(rec.payloads[0], dtype=np.uint8)
        out[f"geom_{tag}_p1"] = np.frombuffer(rec.payloads[1], dtype=np.uint8)
    save("net_frames.npz", **out)


def loader_fixtures(FX, H5, save):
    """The reference loaders with the detector crop, the object box, skip, and an HDF5 scan
    without flat / dark frames, on the deterministic scans of scan_synth.py."""
    sys.path.insert(0, HERE)
    import scan_synth as SS
    tmp = tempfile.mkdtemp(prefix="flexray_crop_")
    SS.write_flexray_scan(tmp)
    out = {}
    for tag, kw in (("s2", dict(sample=2, skip=1)), ("s2k2", dict(sample=2, skip=2)),
                    ("s3", dict(sample=3, skip=1, profile="cwi-flexray-2022-10-28"))):
        kw.setdefault("profile", "cwi-flexray-2019-04-24")
        proj, geom = FX.load_flexray(tmp, crop=True, auto_box=True, verbose=False, **kw)
        out[f"{tag}_proj"], out[f"{tag}_V"], out[f"{tag}_box"] = proj, geom.vectors, geom.box
    out["settings"] = np.array(FX.parse_scan_settings(tmp)["det_tan"])
    for tag, kw in (("nf", dict(sample=2, skip=2, rows="2:30")), ("wf", dict(sample=1, skip=1))):
        files = SS.dxchange_arrays(flat=(tag == "wf"))
        proj, geom = H5.load_dxchange("fake.h5", h5=SS.FakeH5(files), verbose=False, **kw)
        out[f"h5{tag}_proj"], out[f"h5{tag}_angles"] = proj, geom.angles
    save("loaders_device.npz", **out)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    root = args[0] if args else os.environ.get("MINIRECAST_REF")
    if not root or not os.path.isdir(os.path.join(root, "minirecast")):
        sys.exit("usage: make_golden.py PATH-TO-REFERENCE-CHECKOUT [--net-only] "
                 "(or set MINIRECAST_REF): the directory that holds the minirecast package")
    if "--net-only" in sys.argv:                 # only net_frames.npz
        os.environ.setdefault("NUMBA_CACHE_DIR", tempfile.mkdtemp(prefix="numba_cache_"))
        sys.path.insert(0, root)
        net_fixtures(lambda name, **kw: np.savez_compressed(os.path.join(HERE, name), **kw))
    else:
        main(root)
