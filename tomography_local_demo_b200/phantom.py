"""Analytic ellipsoid phantoms and synthetic acquisitions, evaluated with torch in FP64.

The phantom data model is minirecast's (phantom.py:11-37: a table of constant-density
ellipsoids, value, semi-axes, centre, rotation about z, scaled to mm). Every ellipsoid
has an exact line integral, so simulated projections carry no discretisation error.

All evaluation goes through one routine, `chord_integrals`: an ellipsoid maps to the unit
sphere under y = M (x - c), so a line x = p + t w meets it where |M(p - c) + t M w| <= 1,
a quadratic in t whose root distance, times |w| = 1, is the chord length; the integral
is the density times the chord. The chord of the whole line does not depend on where
along the line p sits, so projectors take p on the detector (or the source) directly.
The projectors run batched on any torch device: a full cone acquisition of 600 views of
384 x 486 takes seconds on a GPU. `raw_counts` turns line integrals into uint16 detector
counts with flat / dark fields and Poisson noise.
"""
import numpy as np

# value, a, b, c, x0, y0, z0, phi (deg, about z): the modified 3D Shepp-Logan table of
# minirecast phantom.py:11-22 (a constant: the same phantom must come out)
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


class EllipsoidPhantom:
    """Sum of constant-density ellipsoids, coordinates in mm.

    Per ellipsoid e: density vals[e], centre centers[e] (mm) and the 3x3 map mats[e]
    taking x - centre to the unit sphere (inverse scaled semi-axes after the inverse
    rotation about z)."""

    def __init__(self, scale=1.0, table=MODIFIED_SHEPP_LOGAN):
        self.scale = float(scale)
        self.table = np.asarray(table, float).reshape(-1, 8)
        t = self.table
        phi = np.deg2rad(t[:, 7])
        cos, sin = np.cos(phi), np.sin(phi)
        inv_axes = 1.0 / (self.scale * t[:, 1:4])
        # rows of R^T scaled by the inverse semi-axes: M = diag(1/axes) R^T
        rt = np.zeros((len(t), 3, 3))
        rt[:, 0, 0], rt[:, 0, 1] = cos, sin
        rt[:, 1, 0], rt[:, 1, 1] = -sin, cos
        rt[:, 2, 2] = 1.0
        self.mats = inv_axes[:, :, None] * rt
        self.vals = t[:, 0].copy()
        self.centers = self.scale * t[:, 4:7]

    def _tensors(self, device):
        import torch
        f64 = dict(dtype=torch.float64, device=device)
        return (torch.as_tensor(self.vals, **f64), torch.as_tensor(self.centers, **f64),
                torch.as_tensor(self.mats, **f64))

    def evaluate(self, points):
        """Density at points [..., 3] (mm) -> float64 array [...]."""
        import torch
        pts = torch.as_tensor(np.asarray(points, np.float64))
        vals, cents, mats = self._tensors(pts.device)
        y = torch.einsum("eij,...ej->...ei", mats, pts[..., None, :] - cents)
        inside = (y * y).sum(-1) <= 1.0
        return (inside.double() * vals).sum(-1).numpy()

    def line_integrals(self, starts, dirs):
        """Exact integrals along the lines start + t dir (unit dirs), [..., 3] -> [...]."""
        import torch
        return chord_integrals(self, torch.as_tensor(np.asarray(starts, np.float64)),
                               torch.as_tensor(np.asarray(dirs, np.float64))).numpy()


def chord_integrals(phantom, points, dirs):
    """Line integrals of `phantom` along the full lines through `points` with unit
    directions `dirs` (torch float64 tensors, broadcastable [..., 3]) -> float64 [...]."""
    import torch
    vals, cents, mats = phantom._tensors(points.device)
    shape = torch.broadcast_shapes(points.shape, dirs.shape)[:-1]
    acc = torch.zeros(shape, dtype=torch.float64, device=points.device)
    for e in range(len(vals)):
        a = (points - cents[e]) @ mats[e].T            # foot of the line in sphere space
        b = dirs @ mats[e].T                           # direction in sphere space
        bb = (b * b).sum(-1)
        ab = (a * b).sum(-1)
        # |a + t b|^2 = 1  ->  roots t = (-ab +- sqrt(ab^2 - bb (|a|^2 - 1))) / bb
        disc = ab * ab - bb * ((a * a).sum(-1) - 1.0)
        acc += vals[e] * 2.0 * torch.sqrt(disc.clamp(min=0.0)) / bb
    return acc


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


def project_cone_torch(phantom, geom, device="cuda", views_per_batch=16):
    """Cone-beam line integrals of `phantom` for a ConeVecGeometry (ASTRA vectors: the ray
    of detector pixel (r, c) runs from the source s to d + (c - (C-1)/2) u + (r - (R-1)/2) v).
    FP64 on a torch device; returns a float32 tensor [angles, rows, cols] there."""
    import torch
    dev = torch.device(device)
    R, C = geom.rows, geom.cols
    vec = torch.as_tensor(np.asarray(geom.vectors), dtype=torch.float64, device=dev)
    cc = torch.arange(C, dtype=torch.float64, device=dev) - (C - 1) / 2.0
    rr = torch.arange(R, dtype=torch.float64, device=dev) - (R - 1) / 2.0
    out = torch.empty((len(vec), R, C), dtype=torch.float32, device=dev)
    for k0 in range(0, len(vec), views_per_batch):
        vb = vec[k0:k0 + views_per_batch, None, None, :]          # [b, 1, 1, 12]
        src = vb[..., 0:3]
        pix = vb[..., 3:6] + cc[:, None] * vb[..., 6:9] + rr[:, None, None] * vb[..., 9:12]
        ray = pix - src
        ray = ray / torch.linalg.norm(ray, dim=-1, keepdim=True)
        out[k0:k0 + len(vb)] = chord_integrals(phantom, src, ray).to(torch.float32)
    return out


def project_parallel_torch(phantom, geom, device="cpu"):
    """Parallel-beam line integrals for a ParallelGeometry: the ray of angle th and detector
    pixel (r, c) has direction (cos th, sin th, 0) and passes through u (-sin th, cos th, 0)
    + v (0, 0, 1), u and v the pixel's detector coordinates. Returns float32 [rows, angles,
    cols] (the layout of the reference's projection blocks) on `device`."""
    import torch
    dev = torch.device(device)
    u, v = geom.detector_coords()
    u = torch.as_tensor(u, dtype=torch.float64, device=dev)
    v = torch.as_tensor(v, dtype=torch.float64, device=dev)
    th = torch.as_tensor(np.asarray(geom.angles, np.float64), device=dev)
    zero = torch.zeros_like(th)
    ray = torch.stack([torch.cos(th), torch.sin(th), zero], -1)            # [A, 3]
    across = torch.stack([-torch.sin(th), torch.cos(th), zero], -1)        # [A, 3]
    foot = (u[None, None, :, None] * across[None, :, None, :]
            + v[:, None, None, None] * torch.tensor([0.0, 0.0, 1.0], dtype=torch.float64, device=dev))
    return chord_integrals(phantom, foot, ray[None, :, None, :]).to(torch.float32)


def raw_counts(line_integrals, flat, dark, seed=0):
    """uint16 counts I = Poisson((F - D) exp(-p)) + D, clipped to the uint16 range.
    line_integrals: torch tensor [k, R, C]; flat, dark: torch tensors [R, C]."""
    import torch
    gen = torch.Generator(device=line_integrals.device)
    gen.manual_seed(seed)
    mean = (flat - dark).clamp(min=0) * torch.exp(-line_integrals.double())
    counts = torch.poisson(mean, generator=gen) + dark.double()
    return counts.round().clamp(0, 65535).to(torch.int32)
