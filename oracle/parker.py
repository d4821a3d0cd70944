"""TEST INFRASTRUCTURE ONLY: Parker's short-scan weights (D. L. Parker, "Optimal short scan
convolution reconstruction for fanbeam CT", Med. Phys. 9 (1982) 254-257), restated for a
flat-detector circular cone-beam orbit from the FDK constants of oracle/filter.py: the fan
angle of a column is atan(a / SDD), a its distance along u from the principal point, signed
in the direction of rotation. The reference has no such weights (it warns on short scans,
recon.py:331-332), so these are checked by the sum of conjugate-ray weights and by
reconstructions, not against the reference."""
import numpy as np

from .filter import cone_constants


def parker(vectors, cols):
    """w[v, c] * n d_beta / pi for views `vectors` (first to last = the scanned arc)."""
    K = cone_constants(vectors)
    s, d, u = K["s"], K["d"], K["u"]
    n = len(s)
    orbit = np.sign(np.cross(s[0], s[1])[2])                 # +1: counter-clockwise about z
    start = np.arctan2(s[0, 1], s[0, 0])
    beta = np.mod(orbit * (np.arctan2(s[:, 1], s[:, 0]) - start), 2 * np.pi)
    beta[0] = 0.0
    d_beta = beta[-1] / (n - 1)
    cc = np.arange(cols) - (cols - 1) / 2.0
    out = np.empty((n, cols))
    delta = (beta[-1] - np.pi) / 2
    for k in range(n):
        un = np.linalg.norm(u[k])
        off = d[k] - (s[k] + K["sdd"][k] * K["n"][k])
        a = off @ u[k] / un + cc * un
        side = np.sign(np.cross(-s[k], u[k])[2]) * orbit
        g = side * np.arctan(a / K["sdd"][k])
        b = beta[k]
        w = np.ones(cols)
        rise = b < 2 * (delta - g)
        fall = b > np.pi - 2 * g
        w[rise] = np.sin(np.pi / 4 * b / (delta - g[rise])) ** 2
        w[fall] = np.sin(np.pi / 4 * (np.pi + 2 * delta - b) / (delta + g[fall])) ** 2
        out[k] = w
    return out * (n * d_beta / np.pi)
