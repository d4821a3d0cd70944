"""TEST INFRASTRUCTURE ONLY. CPU restatement of minirecast's SliceReconstructor pipeline
(recon.py:289-519): filter on arrival, arrival-ordered store, on-demand back-projection.

precision="ref"  : the reference's own numerics (float32 store, float64 accumulation,
                   cone filter in float64 cast to float32, parallel filter in float32)
precision="fp64" : the FP64 oracle (float64 filter, float64 store, float64 accumulation)

The geometry argument is duck-typed: `.rows`, `.cols`, `.box` (or None) and either
`.vectors` (cone) or `.angles`, `.pixel_u`, `.pixel_v` (parallel).
"""
import numpy as np

from . import bp as _bp
from . import filter as _f
from . import geometry as _g


class OracleReconstructor:
    def __init__(self, proj, geom, window="shepp-logan", gaussian=0.0, tilt=0.0, precision="ref"):
        self.geom = geom
        self.window = window
        self.gaussian, self.tilt = float(gaussian), float(tilt)
        self.exact64 = precision == "fp64"
        self.kind = "cone" if hasattr(geom, "vectors") else "parallel"
        R, C = geom.rows, geom.cols
        if getattr(geom, "box", None) is not None:
            self.box = np.asarray(geom.box, float)
        elif self.kind == "cone":
            self.box = _g.cone_volume_box(geom.vectors, R, C)
        else:
            self.box = _g.parallel_volume_box(R, C, geom.pixel_u, geom.pixel_v)
        self.n_total = len(geom.vectors) if self.kind == "cone" else len(geom.angles)
        self._q = np.zeros((self.n_total, R, C), np.float64 if self.exact64 else np.float32)
        self._order = np.zeros(self.n_total, np.int64)
        self._received = np.zeros(self.n_total, bool)
        self.n = 0
        self.cor_shift = 0.0
        if self.kind == "cone":
            self._K = _f.cone_constants(geom.vectors)
        if proj is not None:
            for i in range(0, self.n_total, 64):          # recon.py:338-340
                self.add_projections(np.arange(i, min(i + 64, self.n_total)), proj[:, i:i + 64, :])

    def add_projections(self, indices, block):
        """recon.py:346-376."""
        indices = np.asarray(indices, np.int64).ravel()
        block = np.asarray(block, np.float32)
        keep = ~self._received[indices]
        indices, block = indices[keep], block[:, keep, :]
        if len(indices) == 0:
            return self.n
        block = _f.preprocess_apply(block, self.gaussian, self.tilt)
        if self.kind == "parallel":
            filt = _f.parallel_filter_block(block, self.geom.pixel_u, self.window, self.exact64)
        else:
            K = {k: v[indices] for k, v in self._K.items()}
            filt = _f.fdk_filter_block(block, K, self.window, self.exact64)
        n0, n1 = self.n, self.n + len(indices)
        self._q[n0:n1] = filt
        self._order[n0:n1] = indices
        self._received[indices] = True
        self.n = n1
        return self.n

    @property
    def native_pixel(self):
        if self.kind == "parallel":
            return float(self.geom.pixel_u)
        return float(np.linalg.norm(self._K["u"][0]) * self._K["sod"][0] / self._K["sdd"][0])

    def reconstruct_points(self, pts, cor_shift=None):
        """recon.py:405-424."""
        pts = np.ascontiguousarray(np.asarray(pts, np.float64).reshape(-1, 3))
        shift = self.cor_shift if cor_shift is None else float(cor_shift)
        if self.n == 0 or len(pts) == 0:
            return np.zeros(len(pts))
        q = self._q[:self.n]
        order = self._order[:self.n]
        scale = np.pi / self.n
        if self.kind == "parallel":
            a = np.asarray(self.geom.angles, float)[order]
            return _bp.bp_parallel(q, np.cos(a), np.sin(a), self.geom.pixel_u, self.geom.pixel_v,
                                   pts, scale, shift)
        K = {k: v[order] for k, v in self._K.items()}
        D = K["d"] - shift * K["u"] if shift else K["d"]
        return _bp.bp_cone(q, K["s"], D, K["uu"], K["vv"], K["n"], K["sdd"], K["sod"], pts, scale)

    def reconstruct_plane(self, origin, normal, n=256, size=None, zoom=1.0, center=None,
                          cor_shift=None):
        """recon.py:426-440."""
        pts, mask = _g.slice_points(self.box, origin, normal, n, size, zoom, center)
        flat = pts.reshape(-1, 3)
        img = np.zeros(len(flat))
        m = mask.ravel()
        if m.any():
            img[m] = self.reconstruct_points(flat[m], cor_shift)
        return img.reshape(n, n), pts

    def reconstruct_volume(self, voxel=None, maxdim=None):
        """recon.py:442-470 (one slab: the slab split does not change values)."""
        dims, origin, h = _g.volume_points(self.box, voxel, maxdim, self.native_pixel)
        nx, ny, nz = (int(d) for d in dims)
        x, y, z = (origin[i] + h * np.arange(dims[i]) for i in range(3))
        X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
        vals = self.reconstruct_points(np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1))
        return vals.reshape(nx, ny, nz).astype(np.float32), origin, h

    def estimate_cor(self, shifts=None, n=192, z=0.0):
        """recon.py:498-519 - argmax of sum p log p over 128-bin histograms."""
        if shifts is None:
            shifts = np.arange(-3.0, 3.01, 0.25)
        scores = []
        for s in shifts:
            img, _ = self.reconstruct_plane((0.0, 0.0, z), (0.0, 0.0, 1.0), n=n, cor_shift=float(s))
            hist, _ = np.histogram(img[img != 0], bins=128)
            p = hist[hist > 0] / max(hist.sum(), 1)
            scores.append(float(np.sum(p * np.log(p))))
        best = float(shifts[int(np.argmax(scores))])
        self.cor_shift = best
        return best, np.array(scores)
