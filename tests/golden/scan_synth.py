"""Deterministic synthetic scans for the loader fixtures: the same arrays and files come
out on every machine (numpy's seeded generator, uint16 TIFFs written with PIL), so the
reference's loader outputs stored by make_golden.py can be compared with the device
loaders run on files rebuilt from the same seed."""
import os

import numpy as np

SETTINGS = ("Sample name: synthetic skull\nSOD: 300.5 mm\nSDD: 612.25 mm\nVoxel size: 98.7 um\n"
            "ver_tube: 1.25\ntra_tube: -0.5\nver_det: 2.0\ntra_det: 0.75\ntra_obj: 0.3\n"
            "Start angle: 0\nLast angle: 360\nROI (LTRB): 40,60,1880,1470\n")


def flexray_frames(seed=3, views=24, h=120, w=160, n_flat=2, n_dark=3):
    """(scans [views, h, w], flats, darks) uint16: a shadow of a blob that circles the
    rotation axis, Poisson counts between flat ~40000 and dark ~100."""
    rng = np.random.default_rng(seed)
    flat_field = 40000.0 + 2000.0 * rng.random((h, w))
    dark_field = 100.0 + 5.0 * rng.random((h, w))
    rr, cc = np.mgrid[0:h, 0:w].astype(np.float64)
    scans = []
    for i in range(views):
        th = 2.0 * np.pi * i / views
        c0 = 0.5 * w + 0.12 * w * np.cos(th)
        r0 = 0.58 * h + 0.03 * h * np.sin(th)
        q = 1.0 - ((cc - c0) / (0.17 * w)) ** 2 - ((rr - r0) / (0.2 * h)) ** 2
        p = 1.6 * np.sqrt(np.clip(q, 0.0, None))
        counts = rng.poisson((flat_field - dark_field) * np.exp(-p)) + dark_field
        scans.append(np.clip(np.round(counts), 0, 65535).astype(np.uint16))
    flats = [np.clip(np.round(rng.poisson(flat_field - dark_field) + dark_field), 0, 65535).astype(np.uint16)
             for _ in range(n_flat)]
    darks = [np.clip(np.round(dark_field + rng.normal(0.0, 1.0, (h, w))), 0, 65535).astype(np.uint16)
             for _ in range(n_dark)]
    return np.stack(scans), flats, darks


def write_flexray_scan(folder, **kw):
    """A FleX-ray scan folder: scan_*.tif, io*.tif (flats), di*.tif (darks), settings."""
    from PIL import Image
    scans, flats, darks = flexray_frames(**kw)
    os.makedirs(folder, exist_ok=True)
    for i, im in enumerate(scans):
        Image.fromarray(im).save(os.path.join(folder, f"scan_{i:06d}.tif"))
    for i, im in enumerate(flats):
        Image.fromarray(im).save(os.path.join(folder, f"io{i:06d}.tif"))
    for i, im in enumerate(darks):
        Image.fromarray(im).save(os.path.join(folder, f"di{i:06d}.tif"))
    with open(os.path.join(folder, "scan settings.txt"), "w") as f:
        f.write(SETTINGS)
    return scans


def dxchange_arrays(seed=5, views=30, h=34, w=44, flat=True):
    """exchange/* arrays of a parallel-beam scan (uint16 data with some dead pixels)."""
    rng = np.random.default_rng(seed)
    rr, cc = np.mgrid[0:h, 0:w].astype(np.float64)
    data = np.empty((views, h, w), np.uint16)
    for i in range(views):
        th = np.pi * i / views
        c0 = 0.5 * w + 0.2 * w * np.cos(th)
        p = 1.2 * np.exp(-((cc - c0) / (0.15 * w)) ** 2 - ((rr - 0.5 * h) / (0.3 * h)) ** 2)
        data[i] = np.clip(np.round(rng.poisson(5000.0 * np.exp(-p)) + 100.0), 0, 65535)
    data[:, 3, 5] = 0                                       # dead pixel
    out = {"exchange/data": data, "exchange/theta": np.arange(views) * 180.0 / views}
    if flat:
        out["exchange/data_white"] = np.round(rng.normal(5100.0, 40.0, (3, h, w))).astype(np.uint16)
        out["exchange/data_dark"] = np.round(rng.normal(100.0, 2.0, (2, h, w))).astype(np.uint16)
    return out


class FakeH5:
    """Stand-in for the h5py module over a dict of arrays (the reference's tests do the
    same, selftest.py:122-145)."""

    def __init__(self, files):
        self.files = files

    def File(self, path, mode):                  # noqa: N802 (h5py's name)
        files = self.files

        class _F(dict):
            def __enter__(self):
                return self

            def __exit__(self, *a):
                return False

        return _F(files)
