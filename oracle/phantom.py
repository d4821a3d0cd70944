"""TEST INFRASTRUCTURE ONLY. NumPy restatement of minirecast phantom.py (exact ellipsoid
line integrals), used to make test inputs with known answers."""
import numpy as np

# phantom.py:11-22 - modified 3D Shepp-Logan: value, a, b, c, x0, y0, z0, phi (deg, about z)
MODIFIED_SHEPP_LOGAN = np.array([
    [1.0, .6900, .920, .810, 0.00, 0.0000, 0.00, 0],
    [-0.8, .6624, .874, .780, 0.00, -0.0184, 0.00, 0],
    [-0.2, .1100, .310, .220, 0.22, 0.0000, 0.00, -18],
    [-0.2, .1600, .410, .280, -0.22, 0.0000, 0.00, 18],
    [0.1, .2100, .250, .410, 0.00, 0.3500, -0.15, 0],
    [0.1, .0460, .046, .050, 0.00, 0.1000, 0.25, 0],
    [0.1, .0460, .046, .050, 0.00, -0.1000, 0.25, 0],
    [0.1, .0460, .023, .050, -0.08, -0.6050, 0.00, 0],
    [0.1, .0230, .023, .020, 0.00, -0.6060, 0.00, 0],
    [0.1, .0230, .046, .020, 0.06, -0.6050, 0.00, 0],
])


class Phantom:
    """phantom.py:25-70 - sum of constant ellipsoids (mm)."""

    def __init__(self, scale=1.0, table=MODIFIED_SHEPP_LOGAN):
        self.scale = float(scale)
        self.items = []
        for val, a, b, c, x0, y0, z0, phi in np.asarray(table, float):
            p = np.deg2rad(phi)
            rot = np.array([[np.cos(p), -np.sin(p), 0.0], [np.sin(p), np.cos(p), 0.0], [0, 0, 1.0]])
            M = np.diag(1.0 / (np.array([a, b, c]) * self.scale)) @ rot.T
            self.items.append((val, np.array([x0, y0, z0]) * self.scale, M))

    def evaluate(self, points):
        pts = np.asarray(points, dtype=np.float64)
        out = np.zeros(pts.shape[:-1])
        for val, c, M in self.items:
            y = (pts - c) @ M.T
            out += val * (np.sum(y * y, axis=-1) <= 1.0)
        return out

    def line_integrals(self, starts, dirs):
        starts = np.asarray(starts, np.float64)
        dirs = np.asarray(dirs, np.float64)
        out = np.zeros(np.broadcast_shapes(starts.shape, dirs.shape)[:-1])
        for val, c, M in self.items:
            p, q = (starts - c) @ M.T, dirs @ M.T
            qq, pq, pp = (q * q).sum(-1), (p * q).sum(-1), (p * p).sum(-1)
            disc = pq * pq - qq * (pp - 1.0)
            out += val * 2.0 * np.sqrt(np.clip(disc, 0.0, None)) / qq
        return out


def project_parallel(ph, angles, rows, cols, pixel_u, pixel_v):
    """phantom.py:73-83 -> [rows, angles, cols] float32."""
    u = (np.arange(cols) - (cols - 1) / 2.0) * pixel_u
    v = (np.arange(rows) - (rows - 1) / 2.0) * pixel_v
    data = np.empty((rows, len(angles), cols), dtype=np.float32)
    ez = np.array([0.0, 0.0, 1.0])
    for k, th in enumerate(angles):
        d = np.array([np.cos(th), np.sin(th), 0.0])
        eu = np.array([-np.sin(th), np.cos(th), 0.0])
        starts = u[None, :, None] * eu + v[:, None, None] * ez - 10.0 * ph.scale * d
        data[:, k, :] = ph.line_integrals(starts, d)
    return data


def project_cone(ph, vectors, rows, cols):
    """phantom.py:86-98 -> [rows, angles, cols] float32."""
    cc = np.arange(cols) - (cols - 1) / 2.0
    rr = np.arange(rows) - (rows - 1) / 2.0
    data = np.empty((rows, len(vectors), cols), dtype=np.float32)
    for k, vec in enumerate(np.asarray(vectors, float)):
        s, d, u, v = vec[0:3], vec[3:6], vec[6:9], vec[9:12]
        dirs = d + cc[None, :, None] * u + rr[:, None, None] * v - s
        dirs /= np.linalg.norm(dirs, axis=-1, keepdims=True)
        data[:, k, :] = ph.line_integrals(s[None, None, :], dirs)
    return data
