"""Device scan loaders against the reference loaders' own outputs (tests/golden/
loaders_device.npz and loaders.npz, made by make_golden.py on the same synthetic scans):
FleX-ray folders with the shadow crop, the object box, skip and 2x2 / 3x3 binning, and
Data Exchange HDF5 with and without flat / dark frames. The stack differs from the
reference only by the float32 logarithm's last bit; crop, geometry and box are equal."""
import os
import sys

import numpy as np
import pytest
import torch

from conftest import golden
from tomography_local_demo_b200 import SliceReconstructor
from tomography_local_demo_b200 import _native as N
from tomography_local_demo_b200 import loaders as L

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import scan_synth as SS  # noqa: E402

pytestmark = pytest.mark.gpu

FLEX = {"s2": dict(sample=2, skip=1), "s2k2": dict(sample=2, skip=2),
        "s3": dict(sample=3, skip=1, profile="cwi-flexray-2022-10-28")}


@pytest.fixture(scope="module")
def scan_dir(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("flexray"))
    SS.write_flexray_scan(d)
    return d


@pytest.mark.parametrize("tag", list(FLEX))
def test_flexray_matches_reference(cuda, scan_dir, tag):
    g = golden("loaders_device.npz")
    kw = dict(FLEX[tag])
    kw.setdefault("profile", "cwi-flexray-2019-04-24")
    proj, geom = L.load_flexray(scan_dir, crop=True, auto_box=True, verbose=False, chunk=5, **kw)
    want = g[f"{tag}_proj"]
    assert proj.shape == want.shape and proj.dtype == np.float32
    np.testing.assert_allclose(proj, want, rtol=1e-6, atol=1e-6)
    np.testing.assert_array_equal(geom.vectors, g[f"{tag}_V"])
    np.testing.assert_array_equal(geom.box, g[f"{tag}_box"])
    assert (geom.rows, geom.cols) == (want.shape[0], want.shape[2])


def test_flexray_without_crop_matches_reference_fixture(cuda, tmp_path):
    """The older fixture (crop and box off, 2x2 binning, 4 scans of 12 x 18)."""
    from PIL import Image
    g = golden("loaders.npz")
    for i, im in enumerate(g["fx_raw"]):
        Image.fromarray(im).save(str(tmp_path / f"scan_{i:06d}.tif"))
    for i, im in enumerate(g["fx_flat"]):
        Image.fromarray(im).save(str(tmp_path / f"io{i:06d}.tif"))
    for i, im in enumerate(g["fx_dark"]):
        Image.fromarray(im).save(str(tmp_path / f"di{i:06d}.tif"))
    (tmp_path / "scan settings.txt").write_text("SOD: 300\nSDD: 600\nVoxel size: 100\nStart angle: 0\n"
                                                "Last angle: 360\n")
    proj, _ = L.load_flexray(str(tmp_path), sample=2, skip=1, profile="none", auto_box=False, crop=False,
                             verbose=False)
    np.testing.assert_allclose(proj, g["fx_proj"], rtol=1e-6, atol=1e-6)


def test_flexray_device_stack_feeds_the_reconstructor(cuda, scan_dir):
    proj_t, geom = L.load_flexray(scan_dir, sample=2, skip=1, verbose=False, as_tensor=True)
    proj_n, _ = L.load_flexray(scan_dir, sample=2, skip=1, verbose=False)
    assert proj_t.is_cuda
    np.testing.assert_array_equal(proj_t.cpu().numpy(), proj_n)
    a = SliceReconstructor(proj_t, geom, verbose=False).reconstruct_plane((0, 0, 0), (0, 0, 1), n=48)[0]
    b = SliceReconstructor(proj_n, geom, verbose=False).reconstruct_plane((0, 0, 0), (0, 0, 1), n=48)[0]
    np.testing.assert_array_equal(a, b)
    assert np.abs(a).max() > 0


@pytest.mark.parametrize("tag,kw", [("nf", dict(sample=2, skip=2, rows="2:30")), ("wf", dict(sample=1, skip=1))])
def test_dxchange_matches_reference(cuda, tag, kw):
    g = golden("loaders_device.npz")
    files = SS.dxchange_arrays(flat=(tag == "wf"))
    proj, geom = L.load_dxchange("fake.h5", h5=SS.FakeH5(files), verbose=False, **kw)
    want = g[f"h5{tag}_proj"]
    assert proj.shape == want.shape
    np.testing.assert_allclose(proj, want, rtol=1e-6, atol=1e-6)
    np.testing.assert_array_equal(geom.angles, g[f"h5{tag}_angles"])


def test_dxchange_older_fixture_and_float_data(cuda):
    g = golden("loaders.npz")
    files = {"exchange/data": g["h5_data"], "exchange/data_white": g["h5_white"],
             "exchange/data_dark": g["h5_dark"], "exchange/theta": np.arange(8) * 22.5}
    proj, _ = L.load_dxchange("fake.h5", sample=2, h5=SS.FakeH5(files), verbose=False)
    np.testing.assert_allclose(proj, g["h5_proj"], rtol=1e-6, atol=1e-6)
    # float32 counts take the host path of the reference; integral values give the same stack
    ff = dict(files, **{"exchange/data": g["h5_data"].astype(np.float32)})
    pf, _ = L.load_dxchange("fake.h5", sample=2, h5=SS.FakeH5(ff), verbose=False)
    np.testing.assert_allclose(pf, proj, rtol=1e-6, atol=1e-6)


def test_correct_kernel_rejects_bad_arguments(cuda):
    lib = N.load()
    raw = torch.zeros((2, 8, 8), dtype=torch.int16, device="cuda")
    f = torch.zeros((4, 4), dtype=torch.float32, device="cuda")
    out = torch.zeros((4, 2, 4), dtype=torch.float32, device="cuda")
    v = L.ctypes_void

    def call(**over):
        a = dict(k=2, bin=2, flip=1, rows_full=4, row0=0, col0=0, rows=4, cols=4, mode=N.MR_CORRECT_FLEXRAY)
        a.update(over)
        return lib.mr_correct_u16(v(raw.data_ptr()), 64, 8, a["k"], a["bin"], a["flip"], a["rows_full"], a["row0"],
                                  a["col0"], a["rows"], a["cols"], v(f.data_ptr()), v(f.data_ptr()), 4, a["mode"],
                                  v(out.data_ptr()), 8, 4, None)

    assert call() == N.MR_OK
    for bad in (dict(bin=0), dict(bin=17), dict(mode=7), dict(row0=1), dict(cols=5), dict(rows_full=5),
                dict(k=-1)):
        assert call(**bad) == N.MR_ERR_INVALID, bad
    torch.cuda.synchronize()
