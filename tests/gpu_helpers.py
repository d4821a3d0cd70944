"""Helpers of the -m gpu tests: drive the C-ABI kernels directly on given inputs."""
import numpy as np
import torch

from tomography_local_demo_b200 import _native as N
from tomography_local_demo_b200 import recon as R

STORE = {"fp32": (N.MR_F32, torch.float32), "bf16": (N.MR_BF16, torch.bfloat16),
         "fp16": (N.MR_F16, torch.float16)}


class DeviceRing:
    """A filtered-view ring filled from a host stack q [A, R, C] (f32)."""

    def __init__(self, q, maps, kind, store="fp32", qscale=None):
        A, Rr, C = q.shape
        code, tdt = STORE[store]
        pitch = (C + 7) // 8 * 8
        self.dev = torch.device("cuda", 0)
        buf = torch.zeros((A, Rr, pitch), dtype=torch.float32)
        qs = np.ones(A) if qscale is None else np.asarray(qscale, float)
        buf[:, :, :C] = torch.from_numpy((q / qs[:, None, None]).astype(np.float32))
        self.ring = buf.to(tdt).to(self.dev)
        maps = maps.copy()
        maps["qscale"] = qs
        self.views = torch.from_numpy(maps.view(np.uint8).copy()).to(self.dev)
        self.c = R._ring_struct(self.ring, code, kind, Rr, C)
        self.stored = self.ring[:, :, :C].float().cpu().numpy() * qs[:, None, None]

    def run(self, grids, n_out, kernel="staged"):
        out = torch.full((n_out,), float("nan"), dtype=torch.float32, device=self.dev)
        status = torch.zeros(1, dtype=torch.int32, device=self.dev)
        st = torch.cuda.current_stream()
        R.backproject_device(self.c, self.views, grids, out, st, self.dev, kernel=kernel, status=status)
        torch.cuda.synchronize()
        assert int(status.item()) == 0, "device-side wait timed out"
        return out.cpu().numpy().astype(np.float64)

    def points(self, pts, n_views, scale, shift=0.0):
        p = torch.from_numpy(np.ascontiguousarray(pts, np.float32)).to(self.dev)
        g = np.zeros(1, N.GRID_DTYPE)
        g["n_i"], g["n_j"], g["n_k"] = 1, len(pts), 1
        g["flags"] = N.MR_GRID_POINTS
        g["out_stride_j"] = 1
        g["points"] = p.data_ptr()
        g["n_views"], g["scale"], g["cor_shift"] = n_views, scale, shift
        res = self.run(g, len(pts))
        del p
        return res
