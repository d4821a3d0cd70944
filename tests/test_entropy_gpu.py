"""mr_slice_entropy against numpy.histogram + sum(p log p) (recon.py:508-512)."""
import numpy as np
import pytest
import torch

from tomography_local_demo_b200 import _native as N
from tomography_local_demo_b200.recon import ctypes_void

pytestmark = pytest.mark.gpu


def numpy_score(img, bins=128):
    hist, _ = np.histogram(img[img != 0], bins=bins)
    p = hist[hist > 0] / max(hist.sum(), 1)
    return float(np.sum(p * np.log(p)))


def device_scores(imgs, bins=128):
    t = torch.from_numpy(np.ascontiguousarray(imgs, np.float32)).cuda()
    out = torch.empty(len(imgs), dtype=torch.float64, device="cuda")
    n_pix = imgs[0].size
    N.check(N.load().mr_slice_entropy(ctypes_void(t.data_ptr()), len(imgs), n_pix, n_pix, bins,
                                      ctypes_void(out.data_ptr()), None), "entropy")
    return out.cpu().numpy()


def test_entropy_matches_numpy_histogram(cuda):
    rng = np.random.default_rng(0)
    imgs = rng.normal(0.3, 0.2, (9, 96, 96)).astype(np.float32)
    imgs[1][rng.random((96, 96)) < 0.4] = 0.0           # masked-out pixels are zero
    imgs[2] = 0.0                                        # empty histogram -> score 0
    imgs[3] = 0.25                                       # degenerate range
    imgs[4] = np.round(imgs[4] * 8) / 8                  # values exactly on bin edges
    imgs[5, :3, :3] = [[1e-3, -2.0, 5.0], [0, 0, 0], [7.0, 7.0, -2.0]]
    want = np.array([numpy_score(im.astype(np.float64)) for im in imgs])
    got = device_scores(imgs)
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12)
    for bins in (1, 7, 1024):
        np.testing.assert_allclose(device_scores(imgs[:2], bins),
                                   [numpy_score(im.astype(np.float64), bins) for im in imgs[:2]],
                                   rtol=1e-12, atol=1e-12)


def test_entropy_rejects_bad_arguments(cuda):
    t = torch.zeros(4, device="cuda")
    assert N.load().mr_slice_entropy(ctypes_void(t.data_ptr()), 1, 4, 4, 2000, ctypes_void(t.data_ptr()),
                                     None) == N.MR_ERR_INVALID
    assert N.load().mr_slice_entropy(ctypes_void(t.data_ptr()), 1, 2, 4, 8, ctypes_void(t.data_ptr()),
                                     None) == N.MR_ERR_INVALID
