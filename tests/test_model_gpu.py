"""Device Otsu threshold (model.otsu_threshold, model.py:18-29) against the oracle and the
reference's own output: bit-identical thresholds on seeded volumes (zeros, negatives,
ties, a single value, wide ranges, unaligned views), the reference's errors, and the
three C-ABI passes on their own (order statistics = np.sort, histogram = np.histogram,
values on bin edges included)."""
import ctypes

import numpy as np
import pytest
import torch

from conftest import golden
from oracle import model as om
from tomography_local_demo_b200 import _native as N
from tomography_local_demo_b200 import model as M
from tomography_local_demo_b200.recon import ctypes_void as V

pytestmark = pytest.mark.gpu


def _volumes():
    rng = np.random.default_rng(7)
    g = rng.gamma(2.0, 0.1, (64, 64, 64)).astype(np.float32)
    g[g < 0.08] = 0
    yield "gamma", g
    yield "odd", rng.gamma(1.5, 0.2, (129, 67, 33)).astype(np.float32) * (rng.random((129, 67, 33)) > 0.3)
    yield "normal", rng.normal(0.0, 1.0, (50, 40, 30)).astype(np.float32)
    yield "ties", np.round(rng.normal(5.0, 3.0, (40, 40, 40))).astype(np.float32)
    yield "lognormal", rng.lognormal(0.0, 3.0, (33, 33, 33)).astype(np.float32)
    yield "huge", (rng.uniform(-1, 1, (20, 20, 20)) * 1e30).astype(np.float32)
    one = np.zeros((9, 9, 9), np.float32)
    one[4, 4, 4] = 0.25
    yield "single", one
    yield "constant", np.full((7, 8, 9), 3.0, np.float32)
    two = np.zeros(100, np.float32)
    two[[3, 50]] = [-2.0, 7.0]
    yield "two", two


@pytest.mark.parametrize("name,vol", list(_volumes()), ids=[n for n, _ in _volumes()])
def test_threshold_bit_identical_to_oracle(cuda, name, vol):
    want = om.otsu_threshold(vol)
    assert M.otsu_threshold(vol) == want
    t = torch.from_numpy(vol).cuda()
    assert M.otsu_threshold(t) == want
    for bins in (1, 64, 2048):
        assert M.otsu_threshold(t, bins=bins) == om.otsu_threshold(vol, bins=bins)


def test_reference_golden(cuda):
    d = golden("misc.npz")
    assert M.otsu_threshold(d["otsu_vol"]) == float(d["otsu"])


def test_unaligned_views_and_ragged_sizes(cuda):
    rng = np.random.default_rng(3)
    flat = rng.gamma(2.0, 0.1, 4099).astype(np.float32)
    flat[rng.random(4099) < 0.2] = 0
    t = torch.from_numpy(flat).cuda()
    for off in range(4):                          # 0..12 bytes past a 16-byte boundary
        for n in (1, 2, 3, 5, 8, 131, 4095 - off):
            seg = flat[off:off + n]
            if not (seg != 0).any():
                continue
            assert M.otsu_threshold(t[off:off + n]) == om.otsu_threshold(seg), (off, n)


def test_errors_follow_the_reference(cuda):
    with pytest.raises(IndexError):
        M.otsu_threshold(np.zeros((4, 4, 4), np.float32))
    bad = np.ones((4, 4, 4), np.float32)
    bad[1, 1, 1] = np.nan
    with pytest.raises(ValueError, match="not finite"):
        M.otsu_threshold(bad)
    with pytest.raises(ValueError, match="not finite"):
        om.otsu_threshold(bad)
    inf = np.ones(5000, np.float32)
    inf[-10:] = np.inf
    with pytest.raises(ValueError, match="not finite"):
        M.otsu_threshold(inf)
    with pytest.raises(ValueError, match="not finite"):
        om.otsu_threshold(inf)
    with pytest.raises(TypeError):
        M.otsu_threshold(np.ones(8, np.float64))
    with pytest.raises(ValueError):
        M.otsu_threshold(np.ones(8, np.float32), bins=0)


def _ws(dev):
    return torch.empty(int(N.load().mr_volume_workspace_bytes()), dtype=torch.uint8, device=dev)


def test_order_statistics_equal_sorted_values(cuda):
    lib = N.load()
    rng = np.random.default_rng(11)
    for v in (rng.normal(0, 1, 100003).astype(np.float32),
              np.round(rng.normal(0, 2, 5000)).astype(np.float32),
              rng.lognormal(0, 4, 3001).astype(np.float32)):
        t = torch.from_numpy(v).cuda()
        ws = _ws(t.device)
        st = (ctypes.c_uint64 * 3)()
        N.check(lib.mr_volume_stats(V(t.data_ptr()), t.numel(), V(ws.data_ptr()), st, None), "stats")
        nz = v[v != 0]
        assert st[0] == len(nz) and st[1] == 0
        s = np.sort(nz)
        for ranks in ([0], [len(s) - 1], [0, 1, len(s) // 2, len(s) - 1], list(rng.integers(0, len(s), 4))):
            r = (ctypes.c_int64 * len(ranks))(*[int(x) for x in ranks])
            out = torch.empty(4, dtype=torch.float32, device=t.device)
            N.check(lib.mr_volume_select(V(t.data_ptr()), t.numel(), r, len(ranks), st[2] & 0xFFFFFFFF,
                                         st[2] >> 32, V(ws.data_ptr()), V(out.data_ptr()), None), "select")
            np.testing.assert_array_equal(out[:len(ranks)].cpu().numpy(), s[np.asarray(ranks)])


def test_histogram_edges_like_numpy(cuda):
    lib = N.load()
    rng = np.random.default_rng(5)
    edge_vals = (np.arange(9) / 8.0).astype(np.float32)          # exactly on the 8 bins' edges
    v = np.concatenate([edge_vals, rng.uniform(-0.5, 1.5, 20000).astype(np.float32), [0.0]]).astype(np.float32)
    t = torch.from_numpy(v).cuda()
    for lo, hi, bins in ((0.0, 1.0, 8), (0.1, 0.9, 7), (0.25, 0.25, 5), (-0.3, 1.2, 512)):
        first, last = (lo - 0.5, hi + 0.5) if lo == hi else (lo, hi)
        edges = np.linspace(first, last, bins + 1)
        e = torch.from_numpy(edges).cuda()
        h = torch.empty(bins, dtype=torch.int64, device=t.device)
        N.check(lib.mr_volume_histogram(V(t.data_ptr()), t.numel(), V(e.data_ptr()), bins, lo, hi,
                                        V(h.data_ptr()), None), "histogram")
        nz = v[v != 0]
        want, _ = np.histogram(np.clip(nz, np.float64(lo), np.float64(hi)), bins=bins, range=(lo, hi))
        np.testing.assert_array_equal(h.cpu().numpy(), want)


def test_large_volume(cuda):
    rng = np.random.default_rng(1)
    vol = rng.gamma(2.0, 0.1, (256, 256, 256)).astype(np.float32)
    vol[vol < 0.05] = 0
    t = torch.from_numpy(vol).cuda()
    assert M.otsu_threshold(t) == om.otsu_threshold(vol)
