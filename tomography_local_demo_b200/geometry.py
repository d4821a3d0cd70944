"""Scan geometries (the data model of minirecast geometry.py:1-72, kept identical).

Projections are ASTRA-style [rows, angles, cols]. A cone-beam view is an ASTRA
'cone_vec' 12-vector: source (3), detector centre (3), u (3, one column step),
v (3, one row step), all in mm.
"""
from dataclasses import dataclass

import numpy as np


@dataclass
class ParallelGeometry:
    """Parallel beam about the z axis (geometry.py:11-34)."""
    angles: np.ndarray          # radians
    rows: int
    cols: int
    pixel_u: float = 1.0        # mm per detector column
    pixel_v: float = 1.0        # mm per detector row
    box: np.ndarray = None      # half sizes (x, y, z) in mm; None = full field of view

    @property
    def n_angles(self):
        return len(self.angles)

    def detector_coords(self):
        """Detector column / row centres in mm, centred on the detector midpoint."""
        u = self.pixel_u * (np.arange(self.cols) - 0.5 * (self.cols - 1))
        v = self.pixel_v * (np.arange(self.rows) - 0.5 * (self.rows - 1))
        return u, v

    def volume_box(self):
        if self.box is not None:
            return np.asarray(self.box, dtype=float)
        half_u = 0.5 * self.cols * self.pixel_u
        return np.array([half_u, half_u, 0.5 * self.rows * self.pixel_v])


@dataclass
class ConeVecGeometry:
    """Cone beam with one ASTRA cone_vec row per view (geometry.py:37-57)."""
    vectors: np.ndarray         # (n_angles, 12)
    rows: int
    cols: int
    angular_range: float = 2 * np.pi
    box: np.ndarray = None      # half sizes (x, y, z) in mm

    @property
    def n_angles(self):
        return self.vectors.shape[0]

    def volume_box(self):
        """Box seen by the whole detector at the rotation axis (first view)."""
        if self.box is not None:
            return np.asarray(self.box, dtype=float)
        src, det, u, v = (self.vectors[0, 3 * i:3 * i + 3] for i in range(4))
        magnification = np.linalg.norm(det - src) / np.linalg.norm(src)
        half_u = 0.5 * self.cols * np.linalg.norm(u) / magnification
        half_v = 0.5 * self.rows * np.linalg.norm(v) / magnification
        return np.array([half_u, half_u, half_v])


def circular_cone_vectors(n_angles, sod, sdd, rows, cols, pixel, angular_range=2 * np.pi,
                          det_shift_u=0.0):
    """Ideal circular orbit about z (geometry.py:60-72): the source sits at -sod along
    the ray direction (cos a, sin a, 0), the detector centre at sdd - sod, shifted by
    `det_shift_u` pixels along the detector's u axis."""
    a = np.arange(n_angles) * angular_range / n_angles
    ray = np.stack([np.cos(a), np.sin(a), np.zeros_like(a)], axis=1)
    tan = np.stack([-np.sin(a), np.cos(a), np.zeros_like(a)], axis=1)
    vecs = np.zeros((n_angles, 12))
    vecs[:, 0:3] = -sod * ray
    vecs[:, 3:6] = (sdd - sod) * ray + det_shift_u * pixel * tan
    vecs[:, 6:9] = pixel * tan
    vecs[:, 11] = pixel
    return ConeVecGeometry(vecs, rows, cols, angular_range)
