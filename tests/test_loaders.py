"""Host half of the device scan loaders (tomography_local_demo_b200.loaders): the TIFF
frame reader against PIL (the reference's own reader when tifffile is absent), the
scan-settings parser against the reference's value, and the shadow range."""
import os
import struct

import numpy as np
import pytest
from PIL import Image

from conftest import golden
from tomography_local_demo_b200 import loaders as L


@pytest.mark.parametrize("shape", [(1, 1), (7, 13), (120, 160), (300, 517)])
def test_tiff_reader_equals_pil(tmp_path, shape):
    im = np.random.default_rng(shape[0]).integers(0, 65536, shape, dtype=np.uint16)
    fn = str(tmp_path / "a.tif")
    Image.fromarray(im).save(fn)
    with open(fn, "rb") as f:
        assert L._tiff_strips(f) is not None              # the direct path is taken
    np.testing.assert_array_equal(L.read_tiff_u16(fn), np.array(Image.open(fn)))
    buf = np.zeros((2,) + shape, np.uint16)
    L.read_tiff_u16(fn, buf[1])
    np.testing.assert_array_equal(buf[1], im)
    assert not buf[0].any()
    assert L.tiff_shape(fn) == shape
    with pytest.raises(ValueError):
        L.read_tiff_u16(fn, np.zeros((shape[0] + 1, shape[1]), np.uint16))


def _big_endian_tiff(path, im, rows_per_strip):
    """A minimal big-endian ('MM') baseline TIFF with several strips."""
    h, w = im.shape
    strips = [im[r:r + rows_per_strip] for r in range(0, h, rows_per_strip)]
    data = [s.astype(">u2").tobytes() for s in strips]
    n_tags = 9
    ifd_off = 8
    after_ifd = ifd_off + 2 + 12 * n_tags + 4
    offs_off = after_ifd
    cnts_off = offs_off + 4 * len(data)
    data_off = cnts_off + 4 * len(data)
    offsets, pos = [], data_off
    for d in data:
        offsets.append(pos)
        pos += len(d)

    def tag(t, typ, cnt, val):
        if typ == 3 and cnt == 1:
            return struct.pack(">HHIH2x", t, typ, cnt, val)
        return struct.pack(">HHII", t, typ, cnt, val)

    out = b"MM" + struct.pack(">HI", 42, ifd_off) + struct.pack(">H", n_tags)
    out += tag(256, 3, 1, w) + tag(257, 3, 1, h) + tag(258, 3, 1, 16) + tag(259, 3, 1, 1)
    out += tag(262, 3, 1, 1) + tag(273, 4, len(data), offs_off) + tag(277, 3, 1, 1)
    out += tag(278, 3, 1, rows_per_strip) + tag(279, 4, len(data), cnts_off) + struct.pack(">I", 0)
    out += struct.pack(">" + "I" * len(data), *offsets) + struct.pack(">" + "I" * len(data), *[len(d) for d in data])
    out += b"".join(data)
    with open(path, "wb") as f:
        f.write(out)


def test_big_endian_multi_strip_tiff(tmp_path):
    im = np.random.default_rng(1).integers(0, 65536, (37, 29), dtype=np.uint16)
    fn = str(tmp_path / "be.tif")
    _big_endian_tiff(fn, im, rows_per_strip=5)
    np.testing.assert_array_equal(L.read_tiff_u16(fn), im)
    np.testing.assert_array_equal(np.array(Image.open(fn)).astype(np.uint16), im)


def test_compressed_tiff_falls_back_to_pil(tmp_path):
    im = np.random.default_rng(2).integers(0, 4000, (40, 50), dtype=np.uint16)
    fn = str(tmp_path / "c.tif")
    Image.fromarray(im).save(fn, compression="tiff_lzw")
    with open(fn, "rb") as f:
        assert L._tiff_strips(f) is None
    np.testing.assert_array_equal(L.read_tiff_u16(fn), im)
    out = np.empty((40, 50), np.uint16)
    L.read_tiff_u16(fn, out)
    np.testing.assert_array_equal(out, im)


def test_scan_settings_like_the_reference(tmp_path):
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import scan_synth as SS
    (tmp_path / "scan settings.txt").write_text(SS.SETTINGS)
    p = L.parse_scan_settings(str(tmp_path))
    assert p["det_tan"] == float(golden("loaders_device.npz")["settings"])
    assert p["name"] == "synthetic skull" and p["src2obj"] == 300.5 and p["det2obj"] == 612.25 - 300.5
    V = L.cone_vectors(p, [0.0, 90.0], 0.4)
    assert V.shape == (2, 12) and V[0, 11] == 0.4


def test_shadow_range():
    prof = np.zeros(100)
    prof[40:60] = 1.0
    assert L._shadow_range(prof) == (24, 76)
    assert L._shadow_range(np.zeros(10)) == (0, 10)
    prof[0] = prof[99] = 1.0
    assert L._shadow_range(prof) == (0, 100)
