"""Differentiable back-projector: dot-product (adjoint) test, central finite differences
(h = 1e-2 px for the COR shift, 1e-3 deg for the tilt) and a float64 torch-autograd
reference of the same operator; then the gradient-based calibration against the
entropy grid search."""
import math

import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import filter as of
from oracle import geometry as og
from oracle import phantom as oph
from tomography_local_demo_b200 import ConeVecGeometry, SliceReconstructor, circular_cone_vectors
from tomography_local_demo_b200 import _native as N
from tomography_local_demo_b200 import recon as R
from tomography_local_demo_b200.autograd import BackprojectOp, backproject

pytestmark = pytest.mark.gpu


def small_case(A=24, rows=20, cols=28, seed=0):
    rng = np.random.default_rng(seed)
    V = og.circular_cone_vectors(A, 60.0, 100.0, 1.0) + rng.normal(0, 0.01, (A, 12))
    K = R.cone_constants(V)
    maps = R.cone_view_maps(K, rows, cols)
    views = torch.from_numpy(maps.view(np.uint8).copy()).cuda()
    box = og.cone_volume_box(V, rows, cols)
    reqs = [((0.5, -1.0, 1.0), (0.2, 0.3, 1.0), 21, 1.2), ((1, 2, 0), (1.0, 0.1, 0.2), 17, 2.0)]
    grids = np.zeros(len(reqs), N.GRID_DTYPE)
    off = 0
    for r, (o, nrm, n, zm) in enumerate(reqs):
        grids[r] = R.plane_grid(box, o, nrm, n, None, zm, None, 0.0)
        grids[r]["out_offset"] = off
        off += n * n
    op = BackprojectOp(views, N.MR_CONE, rows, cols, grids, off)
    q = torch.from_numpy(rng.normal(0, 1, (A, rows, cols)).astype(np.float32)).cuda()
    q = q + q.roll(1, 2) + q.roll(1, 1)                     # smoother than white noise
    return V, maps, box, reqs, op, q


@pytest.mark.parametrize("shift,tilt", [(0.0, 0.0), (1.3, 0.004)])
def test_dot_product_adjoint(cuda, shift, tilt):
    V, maps, box, reqs, op, q = small_case()
    y = torch.randn(op.n_out, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    Bq = op.forward(q, shift, tilt)
    BTy = op.adjoint(y, shift, tilt)
    lhs = float((Bq.double() * y.double()).sum())
    rhs = float((q.double() * BTy.double()).sum())
    assert abs(lhs - rhs) <= 1e-5 * max(abs(lhs), abs(rhs))


def smooth_field(A, rows, cols, n_out):
    """Low-frequency projections and output weights. The operator is piecewise smooth
    (bilinear taps change at pixel boundaries), so a +/-h difference straddles kinks; with
    white-noise q and y the slope jumps there do not average out and even the exact
    float64 autograd gradient misses the central difference by tens of percent. With
    smooth fields the jumps are small and coherent and the two agree to ~1e-3."""
    k = torch.arange(A, dtype=torch.float64, device="cuda")[:, None, None]
    r = torch.arange(rows, dtype=torch.float64, device="cuda")[None, :, None]
    c = torch.arange(cols, dtype=torch.float64, device="cuda")[None, None, :]
    q = (torch.sin(2 * math.pi * (0.35 * r / rows + 0.45 * c / cols) + 0.7 * k)
         + 0.5 * torch.cos(2 * math.pi * (0.6 * c / cols - 0.25 * r / rows) + 0.3 * k))
    y = 1 + 0.5 * torch.cos(2 * math.pi * 3 * torch.arange(n_out, dtype=torch.float64, device="cuda") / n_out)
    return q.float().contiguous(), y


@pytest.mark.parametrize("seed", [3, 4, 5])
def test_geometry_gradients_match_finite_differences(cuda, seed):
    """Central differences (h = 1e-2 px, 1e-3 deg) of the float64 operator against the
    analytic gradient kernel (an FP32 forward is too noisy for a 1e-3 deg step)."""
    V, maps, box, reqs, op, _ = small_case(A=12, seed=seed)
    q, y = smooth_field(12, 20, 28, op.n_out)
    q64 = q.double()
    grids = op.grids_at(0.0, 0.0)

    def L(s, t):
        f = torch64_reference(q64, maps, grids, torch.tensor(s, dtype=torch.float64, device="cuda"),
                              torch.tensor(t, dtype=torch.float64, device="cuda"), 20, 28)
        return float((f * y).sum())

    for s0, t0 in ((0.4, 0.0), (-1.1, math.radians(0.3))):
        ds, dt = op.grad_geometry(q, y.float(), s0, t0)
        h = 1e-2
        fd_s = (L(s0 + h, t0) - L(s0 - h, t0)) / (2 * h)
        ht = math.radians(1e-3)
        fd_t = (L(s0, t0 + ht) - L(s0, t0 - ht)) / (2 * ht)
        assert abs(float(ds) - fd_s) <= 1e-2 * abs(fd_s) + 1e-6, (seed, s0, float(ds), fd_s)
        assert abs(float(dt) - fd_t) <= 1e-2 * abs(fd_t) + 1e-6, (seed, s0, float(dt), fd_t)


def torch64_reference(q64, maps, grids, shift, tilt, rows, cols):
    """The same operator in float64 torch (autograd-capable): per view, tilt/shift applied
    to the projective map, bilinear with zeros outside, weight 1/den^2, scale pi/n."""
    A = q64.shape[0]
    cc, cr = (cols - 1) / 2.0, (rows - 1) / 2.0
    c, s = torch.cos(tilt), torch.sin(tilt)
    outs = []
    for g in grids:
        n_i, n_j = int(g["n_i"]), int(g["n_j"])
        i, j = torch.meshgrid(torch.arange(n_i, dtype=torch.float64), torch.arange(n_j, dtype=torch.float64),
                              indexing="ij")
        P = (torch.tensor(g["origin"].astype(np.float64)) + i[..., None] * torch.tensor(g["step_i"].astype(np.float64))
             + j[..., None] * torch.tensor(g["step_j"].astype(np.float64))).reshape(-1, 3).cuda()
        Ph = torch.cat([P, torch.ones(len(P), 1, dtype=torch.float64, device="cuda")], 1)
        acc = torch.zeros(len(P), dtype=torch.float64, device="cuda")
        for k in range(A):
            pu = torch.tensor(maps["pu"][k].astype(np.float64), device="cuda")
            pv = torch.tensor(maps["pv"][k].astype(np.float64), device="cuda")
            pw = torch.tensor(maps["pw"][k].astype(np.float64), device="cuda")
            uv = float(maps["uv"][k])
            pu2 = c * pu + s * pv + (cc * (1 - c) - cr * s + shift) * pw
            pv2 = -s * pu + c * pv + (cr * (1 - c) + cc * s + shift * uv) * pw
            den = Ph @ pw
            col, row = (Ph @ pu2) / den, (Ph @ pv2) / den
            r0, c0 = torch.floor(row).detach(), torch.floor(col).detach()
            fr, fc = row - r0, col - c0
            val = 0
            for dr, wr in ((0, 1 - fr), (1, fr)):
                for dc, wc in ((0, 1 - fc), (1, fc)):
                    ri, ci = (r0 + dr).long(), (c0 + dc).long()
                    ok = (ri >= 0) & (ri < rows) & (ci >= 0) & (ci < cols)
                    tap = q64[k][ri.clamp(0, rows - 1), ci.clamp(0, cols - 1)] * ok
                    val = val + wr * wc * tap
            acc = acc + val / den ** 2
        mask = torch.from_numpy(_mask(g)).cuda().reshape(-1)
        outs.append(acc * (math.pi / A) * mask)
    return torch.cat(outs)


def _mask(g):
    n = int(g["n_i"])
    a = (np.arange(n) - g["mask_half"]) * g["mask_delta"]
    ok = np.ones((n, n), bool)
    for e in range(3):
        p = (g["mask_c"][e] + a[None, :] * g["mask_ej"][e]) + a[:, None] * g["mask_ei"][e]
        ok &= np.abs(p) <= g["box"][e]
    return ok


def test_backward_matches_float64_autograd(cuda):
    V, maps, box, reqs, op, q = small_case(A=12, seed=5)
    shift0, tilt0 = 0.7, math.radians(0.4)
    y = torch.randn(op.n_out, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    # ours
    qa = q.clone().requires_grad_(True)
    sa = torch.tensor(shift0, dtype=torch.float64, requires_grad=True)
    ta = torch.tensor(tilt0, dtype=torch.float64, requires_grad=True)
    f = backproject(qa, sa, ta, op)
    (f.double() * y.double()).sum().backward()
    # float64 reference
    q64 = q.double().clone().requires_grad_(True)
    s64 = torch.tensor(shift0, dtype=torch.float64, device="cuda", requires_grad=True)
    t64 = torch.tensor(tilt0, dtype=torch.float64, device="cuda", requires_grad=True)
    f64 = torch64_reference(q64, maps, op.grids_at(0.0, 0.0), s64, t64, 20, 28)
    (f64 * y.double()).sum().backward()
    assert rel_l2(f.detach().cpu().numpy(), f64.detach().cpu().numpy()) < 1e-5
    assert rel_l2(qa.grad.cpu().numpy(), q64.grad.cpu().numpy()) < 1e-5
    assert abs(float(sa.grad) - float(s64.grad)) <= 1e-3 * abs(float(s64.grad))
    assert abs(float(ta.grad) - float(t64.grad)) <= 1e-3 * abs(float(t64.grad))


def test_gradient_calibration_matches_grid_search(cuda):
    """Cone geometry with a seeded +1.7 px rotation-centre error (det_shift_u = -1.7, as in
    minirecast selftest.py:89-92): the gradient calibration lands within 0.1 px of the
    entropy grid-search optimum (refined on a 0.05 px grid around the +/-3 px search)."""
    ph = oph.Phantom(scale=30.0)
    rows, cols = 64, 96
    moved = circular_cone_vectors(120, 300.0, 500.0, rows, cols, 1.0, det_shift_u=-1.7)
    proj = oph.project_cone(ph, moved.vectors, rows, cols)
    geom = circular_cone_vectors(120, 300.0, 500.0, rows, cols, 1.0)
    rec = SliceReconstructor(proj, geom, verbose=False)
    coarse, _ = rec.estimate_cor(n=96, verbose=False)
    fine_shifts = np.arange(coarse - 0.3, coarse + 0.301, 0.05)
    fine = float(fine_shifts[np.argmax(rec.cor_scores(fine_shifts, n=96))])
    shift, tilt, hist = rec.calibrate(shift0=0.0, n=96, fit_tilt=False)
    assert abs(shift - fine) <= 0.1, (shift, fine, coarse, hist[-3:])
    assert abs(shift - 1.7) <= 0.25
