"""Analytic ellipsoid phantoms (the data model of minirecast phantom.py) and synthetic
acquisitions.

Every ellipsoid has an exact line integral, so simulated projections carry no
discretisation error. Besides the reference's NumPy API (EllipsoidPhantom,
project_parallel, project_cone), `project_cone_torch` evaluates the same integrals in
FP64 with torch on any device, which makes full-size cone acquisitions (600 views of
384 x 486) take seconds on a GPU, and `raw_counts` turns line integrals into uint16
detector counts with flat/dark fields and Poisson noise.
"""
import numpy as np

# value, a, b, c, x0, y0, z0, phi (deg, about z) - modified 3D Shepp-Logan (phantom.py:11-22)
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


def _frames(table, scale):
    """(values, centres, M) with M (x - c) mapping each ellipsoid to the unit sphere."""
    vals, cents, mats = [], [], []
    for v, a, b, c, x0, y0, z0, phi in np.asarray(table, float):
        p = np.deg2rad(phi)
        rot = np.array([[np.cos(p), -np.sin(p), 0.0], [np.sin(p), np.cos(p), 0.0], [0.0, 0.0, 1.0]])
        mats.append(np.diag(1.0 / (scale * np.array([a, b, c]))) @ rot.T)
        vals.append(v)
        cents.append(scale * np.array([x0, y0, z0]))
    return np.array(vals), np.array(cents), np.array(mats)


class EllipsoidPhantom:
    """Sum of constant-density ellipsoids, coordinates in mm (phantom.py:40-70)."""

    def __init__(self, scale=1.0, table=MODIFIED_SHEPP_LOGAN):
        self.scale = float(scale)
        self.table = np.asarray(table, float)
        self.vals, self.centers, self.mats = _frames(self.table, self.scale)

    def evaluate(self, points):
        pts = np.asarray(points, dtype=np.float64)
        out = np.zeros(pts.shape[:-1])
        for v, c, M in zip(self.vals, self.centers, self.mats):
            y = (pts - c) @ M.T
            out += v * (np.einsum("...i,...i->...", y, y) <= 1.0)
        return out

    def line_integrals(self, starts, dirs):
        """Exact integrals along start + t dir (unit dirs), shape (..., 3) -> (...)."""
        starts = np.asarray(starts, np.float64)
        dirs = np.asarray(dirs, np.float64)
        out = np.zeros(np.broadcast_shapes(starts.shape, dirs.shape)[:-1])
        for v, c, M in zip(self.vals, self.centers, self.mats):
            p, q = (starts - c) @ M.T, dirs @ M.T
            qq = np.einsum("...i,...i->...", q, q)
            pq = np.einsum("...i,...i->...", p, q)
            pp = np.einsum("...i,...i->...", p, p)
            out += v * 2.0 * np.sqrt(np.clip(pq * pq - qq * (pp - 1.0), 0.0, None)) / qq
        return out


def random_ellipsoids(n, seed, mu_range=(0.01, 0.2), axes_range=(2.0, 25.0), radius=30.0):
    """Table of n seeded random ellipsoids (attenuation per mm, semi-axes and centres in
    mm), each inside a sphere of `radius` mm about the origin; rotation about z only,
    as the table format supports."""
    rng = np.random.default_rng(seed)
    rows = []
    while len(rows) < n:
        ax = rng.uniform(*axes_range, 3)
        r_c = radius - ax.max()
        if r_c <= 0:
            continue
        d = rng.normal(size=3)
        c = d / np.linalg.norm(d) * r_c * rng.uniform(0, 1) ** (1 / 3)
        rows.append([rng.uniform(*mu_range), *ax, *c, rng.uniform(0, 180)])
    return np.array(rows)


def project_parallel(phantom, geom):
    """Analytic parallel-beam projections [rows, angles, cols] float32 (phantom.py:73-83)."""
    u, v = geom.detector_coords()
    data = np.empty((geom.rows, len(geom.angles), geom.cols), dtype=np.float32)
    ez = np.array([0.0, 0.0, 1.0])
    for k, th in enumerate(geom.angles):
        d = np.array([np.cos(th), np.sin(th), 0.0])
        eu = np.array([-np.sin(th), np.cos(th), 0.0])
        starts = u[None, :, None] * eu + v[:, None, None] * ez - 10.0 * phantom.scale * d
        data[:, k, :] = phantom.line_integrals(starts, d)
    return data


def project_cone(phantom, geom):
    """Analytic cone-beam projections [rows, angles, cols] float32 (phantom.py:86-98)."""
    R, C = geom.rows, geom.cols
    cc = np.arange(C) - (C - 1) / 2.0
    rr = np.arange(R) - (R - 1) / 2.0
    data = np.empty((R, geom.n_angles, C), dtype=np.float32)
    for k, vec in enumerate(geom.vectors):
        s, d, u, v = vec[0:3], vec[3:6], vec[6:9], vec[9:12]
        dirs = d + cc[None, :, None] * u + rr[:, None, None] * v - s
        dirs /= np.linalg.norm(dirs, axis=-1, keepdims=True)
        data[:, k, :] = phantom.line_integrals(s[None, None, :], dirs)
    return data


def project_cone_torch(phantom, geom, device="cuda", views_per_batch=16):
    """The same integrals as project_cone, FP64 on a torch device.
    Returns a float32 tensor [angles, rows, cols] on that device."""
    import torch
    dev = torch.device(device)
    R, C = geom.rows, geom.cols
    V = torch.as_tensor(np.asarray(geom.vectors), dtype=torch.float64, device=dev)
    cc = torch.arange(C, dtype=torch.float64, device=dev) - (C - 1) / 2.0
    rr = torch.arange(R, dtype=torch.float64, device=dev) - (R - 1) / 2.0
    vals = torch.as_tensor(phantom.vals, dtype=torch.float64, device=dev)
    cents = torch.as_tensor(phantom.centers, dtype=torch.float64, device=dev)
    mats = torch.as_tensor(phantom.mats, dtype=torch.float64, device=dev)
    out = torch.empty((len(V), R, C), dtype=torch.float32, device=dev)
    for k0 in range(0, len(V), views_per_batch):
        vb = V[k0:k0 + views_per_batch]
        s, d, u, v = vb[:, 0:3], vb[:, 3:6], vb[:, 6:9], vb[:, 9:12]
        pix = (d[:, None, None, :] + cc[None, None, :, None] * u[:, None, None, :]
               + rr[None, :, None, None] * v[:, None, None, :])
        dirs = pix - s[:, None, None, :]
        dirs = dirs / torch.linalg.norm(dirs, dim=-1, keepdim=True)
        acc = torch.zeros(dirs.shape[:-1], dtype=torch.float64, device=dev)
        for e in range(len(vals)):
            M = mats[e]
            p = (s - cents[e]) @ M.T                       # [b, 3]
            q = dirs @ M.T                                 # [b, R, C, 3]
            qq = (q * q).sum(-1)
            pq = (q * p[:, None, None, :]).sum(-1)
            pp = (p * p).sum(-1)[:, None, None]
            acc += vals[e] * 2.0 * torch.sqrt(torch.clamp(pq * pq - qq * (pp - 1.0), min=0.0)) / qq
        out[k0:k0 + len(vb)] = acc.to(torch.float32)
    return out


def raw_counts(line_integrals, flat, dark, seed=0):
    """uint16 counts I = Poisson((F - D) exp(-p)) + D, clipped to the uint16 range.
    line_integrals: torch tensor [k, R, C]; flat, dark: torch tensors [R, C]."""
    import torch
    gen = torch.Generator(device=line_integrals.device)
    gen.manual_seed(seed)
    mean = (flat - dark).clamp(min=0) * torch.exp(-line_integrals.double())
    counts = torch.poisson(mean, generator=gen) + dark.double()
    return counts.round().clamp(0, 65535).to(torch.int32)
