"""Differentiable back-projection f = B(q; cor_shift, tilt).

B is the FDK/FBP back-projection of minirecast recon.py:156-219 (bilinear, zero outside
the detector, (SOD/L)^2 weight, scale pi/n) over any set of sample grids (slices,
windows, volumes, point lists). The backward pass is hand-written:
  * dL/dq      = B^T dL/df  - the matched forward projector (mr_project_adjoint), the
                 exact transpose of the bilinear back-projection;
  * dL/dshift, dL/dtilt     - mr_bp_grad_geom, from the analytic derivative of the
                 bilinear interpolant with respect to the detector coordinates.
Geometry is recomputed in the backward kernels from the per-view maps; nothing from the
forward pass besides its inputs is kept. The tilt is an in-plane rotation (radians) of
the detector coordinates about the detector centre, applied before the COR shift.

This has no counterpart in the reference, whose back-projector is not differentiable.
"""
import math

import numpy as np
import torch

from . import _native as N
from .recon import _ring_struct, _struct_tensor, ctypes_void

_CODES = {torch.float32: N.MR_F32, torch.bfloat16: N.MR_BF16, torch.float16: N.MR_F16}


class BackprojectOp:
    """Geometry and sample grids of one differentiable back-projection.

    views   : device uint8 tensor of mr_view records (one per stored view, slot order)
    kind    : N.MR_CONE or N.MR_PARALLEL
    rows, cols : detector size
    grids   : numpy GRID_DTYPE records; outputs are laid out by their out_offset/strides
    n_out   : length of the flat output
    n_views : views used (default: all records in `views`)
    scale   : factor of the sum over views (default pi / n_views, the FBP scale; 1 gives the
              plain back-projection A^T of the matched forward projector A = B^T)
    """

    def __init__(self, views, kind, rows, cols, grids, n_out, n_views=None, scale=None):
        self.scale = scale              # None: the FBP scale pi / n_views; else this factor
        self.views = views
        self.kind = kind
        self.rows, self.cols = int(rows), int(cols)
        self.grids = np.ascontiguousarray(grids, dtype=N.GRID_DTYPE).copy()
        self.n_out = int(n_out)
        self.n_views = int(n_views if n_views is not None else views.numel() // N.VIEW_DTYPE.itemsize)
        self.device = views.device

    def grids_at(self, shift, tilt):
        g = self.grids.copy()
        g["cor_shift"] = shift
        g["tilt"] = tilt
        if tilt != 0.0:
            g["tilt_cos"], g["tilt_sin"] = math.cos(tilt), math.sin(tilt)
        else:
            g["tilt_cos"], g["tilt_sin"] = 0.0, 0.0
        g["n_views"] = self.n_views
        g["view_begin"], g["accumulate"] = 0, 0      # slots [0, n_views), written (not added)
        if self.scale is not None:
            g["scale"] = self.scale
        else:
            g["scale"] = math.pi / self.n_views if self.n_views else 0.0
        return g

    def _ring(self, q):
        if q.dim() != 3 or q.shape[1] != self.rows or q.shape[2] < self.cols:
            raise ValueError(f"q must be [views, {self.rows}, >= {self.cols}], got {tuple(q.shape)}")
        if q.shape[0] < self.n_views:
            raise ValueError("q holds fewer views than the operator uses")
        if not q.is_contiguous():
            raise ValueError("q must be contiguous")
        return _ring_struct(q, _CODES[q.dtype], self.kind, self.rows, self.cols)

    def forward(self, q, shift=0.0, tilt=0.0):
        """B q with the coordinate arithmetic of the backward kernels (mr_backproject_matched)."""
        out = torch.zeros(self.n_out, dtype=torch.float32, device=self.device)
        grids = self.grids_at(shift, tilt)
        g_dev, t_dev = self._tiles(grids)
        st = torch.cuda.current_stream(self.device)
        v = ctypes_void
        N.check(N.load().mr_backproject_matched(self._ring(q), v(self.views.data_ptr()), v(g_dev.data_ptr()),
                                                v(t_dev.data_ptr()), t_dev.numel() // N.TILE_DTYPE.itemsize,
                                                v(out.data_ptr()), v(st.cuda_stream)), "mr_backproject_matched")
        return out

    def _tiles(self, grids):
        return _struct_tensor(grids, self.device), _struct_tensor(N.plan_tiles(grids), self.device)

    def adjoint(self, gout, shift=0.0, tilt=0.0, shape=None):
        """B^T gout as an f32 tensor of `shape` ([views, rows, pitch])."""
        shape = shape or (self.n_views, self.rows, self.cols)
        gq = torch.zeros(shape, dtype=torch.float32, device=self.device)
        grids = self.grids_at(shift, tilt)
        g_dev, t_dev = self._tiles(grids)
        st = torch.cuda.current_stream(self.device)
        gout = gout.to(torch.float32).contiguous()
        ring = _ring_struct(gq, N.MR_F32, self.kind, self.rows, self.cols)
        v = ctypes_void
        N.check(N.load().mr_project_adjoint(ring, v(self.views.data_ptr()), v(g_dev.data_ptr()),
                                            v(t_dev.data_ptr()), t_dev.numel() // N.TILE_DTYPE.itemsize,
                                            v(gout.data_ptr()), v(st.cuda_stream)), "mr_project_adjoint")
        return gq

    def grad_geometry(self, q, gout, shift=0.0, tilt=0.0):
        """(d<gout, B q>/dshift, d<gout, B q>/dtilt) summed over the grids."""
        grids = self.grids_at(shift, tilt)
        g_dev, t_dev = self._tiles(grids)
        d = torch.zeros(2 * len(grids), dtype=torch.float64, device=self.device)
        st = torch.cuda.current_stream(self.device)
        gout = gout.to(torch.float32).contiguous()
        v = ctypes_void
        N.check(N.load().mr_bp_grad_geom(self._ring(q), v(self.views.data_ptr()), v(g_dev.data_ptr()),
                                         v(t_dev.data_ptr()), t_dev.numel() // N.TILE_DTYPE.itemsize,
                                         v(gout.data_ptr()), v(d.data_ptr()), v(st.cuda_stream)),
                "mr_bp_grad_geom")
        d = d.view(-1, 2).sum(0)
        return d[0], d[1]


class _Backproject(torch.autograd.Function):
    @staticmethod
    def forward(ctx, q, shift, tilt, op):
        ctx.op = op
        ctx.save_for_backward(q, shift, tilt)
        return op.forward(q, float(shift), float(tilt))

    @staticmethod
    def backward(ctx, gout):
        q, shift, tilt = ctx.saved_tensors
        op = ctx.op
        s, t = float(shift), float(tilt)
        gq = gs = gt = None
        if ctx.needs_input_grad[0]:
            gq = op.adjoint(gout, s, t, tuple(q.shape)).to(q.dtype)
        if ctx.needs_input_grad[1] or ctx.needs_input_grad[2]:
            ds, dt = op.grad_geometry(q, gout, s, t)
            gs = ds.to(shift.dtype).to(shift.device).reshape(shift.shape)
            gt = dt.to(tilt.dtype).to(tilt.device).reshape(tilt.shape)
        return gq, gs, gt, None


def backproject(q, shift, tilt, op):
    """Differentiable B(q; shift, tilt) -> flat f32 tensor of op.n_out samples.
    q: [views, rows, >= cols] device tensor (f32 for a q-gradient); shift, tilt: 0-dim
    tensors (detector columns, radians)."""
    shift = torch.as_tensor(shift, dtype=torch.float64)
    tilt = torch.as_tensor(tilt, dtype=torch.float64)
    return _Backproject.apply(q, shift, tilt, op)


# ------------------------------------------------------------------ calibration
def soft_neg_entropy(img, lo, hi, bins=128, bandwidth=1.0):
    """Differentiable counterpart of the estimate_cor score sum(p log p) (recon.py:508-512):
    a histogram of the non-zero pixels with Gaussian-kernel bin membership (width
    `bandwidth` bins) over the fixed range [lo, hi]."""
    x = img[img != 0]
    centres = lo + (torch.arange(bins, dtype=x.dtype, device=x.device) + 0.5) * (hi - lo) / bins
    h = (hi - lo) / bins * bandwidth
    w = torch.exp(-0.5 * ((x[:, None] - centres[None, :]) / h) ** 2)
    w = w / w.sum(1, keepdim=True).clamp_min(1e-30)
    p = w.sum(0) / x.numel()
    p = p.clamp_min(1e-30)
    return (p * torch.log(p)).sum()
