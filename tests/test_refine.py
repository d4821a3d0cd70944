"""Least-squares refinement of few-view live slices: the NumPy restatement (oracle/ls.py)
on CPU, and the CUDA path (SliceReconstructor.refine_slice_ls: matched forward projector
+ back-projection in CGLS) against it on the GPU. Case: a parallel-beam Shepp-Logan scan
of which only every 9th of 180 views has arrived, axial slice on a detector row."""
import numpy as np
import pytest

from conftest import rel_l2
from oracle import ls as ols
from oracle import phantom as oph
from tomography_local_demo_b200 import ParallelGeometry, SliceReconstructor
from tomography_local_demo_b200.recon import slice_points

R, C, A_TOTAL, ROW, N = 64, 96, 180, 37, 64


@pytest.fixture(scope="module")
def scan():
    ph = oph.Phantom(scale=40.0)
    angles = np.arange(A_TOTAL) * np.pi / A_TOTAL
    proj = oph.project_parallel(ph, angles, R, C, 1.0, 1.0)           # [R, A, C]
    geom = ParallelGeometry(angles, R, C, 1.0, 1.0)
    z = ROW - (R - 1) / 2.0                                           # on a detector row
    pts, mask = slice_points(geom.volume_box(), (0.0, 0.0, z), (0.0, 0.0, 1.0), N)
    return ph, angles, proj, geom, z, pts, mask


def test_oracle_refinement_reduces_error_of_few_view_fbp(scan):
    ph, angles, proj, geom, z, pts, mask = scan
    few = np.arange(0, A_TOTAL, 9)
    P = pts[mask]
    x0, x, hist = ols.refine_parallel_axial(proj[ROW, few, :], angles[few], 1.0, P, 5)
    truth = ph.evaluate(P)
    e0, e5 = rel_l2(x0, truth), rel_l2(x, truth)
    assert e5 < 0.85 * e0, (e0, e5)
    assert all(b <= a * (1 + 1e-12) for a, b in zip(hist, hist[1:]))   # CGLS residuals never grow


@pytest.mark.gpu
def test_refine_slice_ls_matches_oracle(cuda, scan):
    ph, angles, proj, geom, z, pts, mask = scan
    few = np.arange(0, A_TOTAL, 9)
    rec = SliceReconstructor(None, geom, verbose=False, keep_projections=True)
    rec.add_projections(few, proj[:, few, :])
    fbp, _ = rec.reconstruct_plane((0.0, 0.0, z), (0.0, 0.0, 1.0), n=N)
    img, hist = rec.refine_slice_ls((0.0, 0.0, z), (0.0, 0.0, 1.0), n=N, iters=5)
    x0, x, hist64 = ols.refine_parallel_axial(proj[ROW, few, :], angles[few], 1.0, pts[mask], 5)
    assert np.array_equal(img == 0, ~mask)                            # zero outside the box
    assert rel_l2(fbp[mask], x0) < 1e-4                               # the FBP start
    assert rel_l2(img[mask], x) < 2e-3                                # FP32 CGLS vs FP64 CGLS
    assert np.allclose(np.array(hist) / hist[0], np.array(hist64) / hist64[0], rtol=2e-3, atol=1e-6)
    truth = ph.evaluate(pts[mask])
    assert rel_l2(img[mask], truth) < 0.85 * rel_l2(fbp[mask], truth)


@pytest.mark.gpu
def test_refine_needs_kept_projections(cuda, scan):
    ph, angles, proj, geom, z, pts, mask = scan
    rec = SliceReconstructor(None, geom, verbose=False)
    rec.add_projections(np.arange(0, A_TOTAL, 9), proj[:, ::9, :])
    with pytest.raises(RuntimeError):
        rec.refine_slice_ls((0.0, 0.0, z), (0.0, 0.0, 1.0), n=N)
