"""TEST INFRASTRUCTURE ONLY. Least-squares refinement of a few-view axial slice, restated
in NumPy as the checker of SliceReconstructor.refine_slice_ls.

The reference (minirecast) has no iterative refinement; this restates the method the
CUDA path implements, built from the reference's parallel-beam geometry (recon.py:175-191:
col = (-x sin t + y cos t) / pixel_u + (C - 1) / 2, bilinear taps outside the detector
contribute 0) and its FBP (recon.py:58-64 filter_rows with tau = pixel_u, scale pi / n):

  A     dense matrix of the bilinear splat of the slice's in-box samples onto one detector
        row of every received view (the transpose of the bilinear back-projection);
  x0    FBP slice = pi / n * A^T (filtered row);
  c     least-squares scale with A x0 ~ c p on the detector pixels the slice reaches
        (splat weight A 1 above 1e-3 of its maximum);
  CGLS  on min ||A x - c p||^2 from x0.
"""
import numpy as np

from . import filter as of


def splat_matrix(points, angles, cols, pixel_u):
    """A[(view, col), sample] for in-box sample points (M, 3) lying on a detector row."""
    A = np.zeros((len(angles) * cols, len(points)))
    for i, th in enumerate(angles):
        col = (-points[:, 0] * np.sin(th) + points[:, 1] * np.cos(th)) / pixel_u + (cols - 1) / 2.0
        c0 = np.floor(col).astype(np.int64)
        fc = col - c0
        for dc, w in ((0, 1.0 - fc), (1, fc)):
            cc = c0 + dc
            ok = (cc >= 0) & (cc < cols)
            np.add.at(A, (i * cols + cc[ok], np.nonzero(ok)[0]), w[ok])
    return A


def refine_parallel_axial(row_proj, angles, pixel_u, points, iters, window="shepp-logan"):
    """row_proj: [views, cols] line integrals of the detector row the slice lies on.
    Returns (x0 FBP, x refined, residual norms), all float64, over `points`."""
    V, C = row_proj.shape
    A = splat_matrix(points, angles, C, pixel_u)
    q = of.filter_rows(row_proj[None].astype(np.float64), pixel_u, window, exact64=True)[0]
    x0 = (A.T @ q.reshape(-1)) * np.pi / V
    p = row_proj.reshape(-1).astype(np.float64)
    w1 = A @ np.ones(A.shape[1])
    A = A * (w1 > 1e-3 * w1.max())[:, None]          # detector pixels the slice reaches
    Ax = A @ x0
    pm = p * (w1 > 1e-3 * w1.max())
    b = (Ax @ pm) / max(pm @ pm, 1e-300) * pm
    x = x0.copy()
    r = b - Ax
    s = A.T @ r
    d = s.copy()
    gamma = s @ s
    hist = [float(np.linalg.norm(r))]
    for _ in range(iters):
        qv = A @ d
        alpha = gamma / (qv @ qv)
        x = x + alpha * d
        r = r - alpha * qv
        s = A.T @ r
        gamma_new = s @ s
        d = s + gamma_new / gamma * d
        gamma = gamma_new
        hist.append(float(np.linalg.norm(r)))
    return x0, x, hist
