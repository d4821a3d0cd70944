"""Parker short-scan weights (recon.parker_weights): the product's formulation (fan angles
from the geometry vectors) against the oracle's (from the FDK constants), the defining
property (the two measurements of a ray weigh 1 together), and the errors."""
import numpy as np
import pytest

from oracle.parker import parker
from tomography_local_demo_b200 import circular_cone_vectors
from tomography_local_demo_b200.recon import parker_weights


def _short(n=200, extra=0.40, shift=0.0, cols=64, reverse=False):
    g = circular_cone_vectors(n, 300.0, 600.0, 48, cols, 3.0, angular_range=np.pi + extra, det_shift_u=shift)
    return g.vectors[::-1].copy() if reverse else g.vectors


@pytest.mark.parametrize("kw", [dict(), dict(shift=1.5), dict(reverse=True), dict(extra=0.9), dict(cols=65)])
def test_weights_equal_oracle(kw):
    V = _short(**kw)
    cols = kw.get("cols", 64)
    np.testing.assert_allclose(parker_weights(V, cols), parker(V, cols), rtol=0, atol=1e-12)


def test_conjugate_rays_weigh_one():
    n, cols = 400, 64
    V = _short(n=n, extra=0.40, cols=cols)
    w = parker_weights(V, cols)
    scale = w.max()                                      # n d_beta / pi (plateau of 1)
    d_beta = (np.pi + 0.40) / n
    gamma = np.arctan((np.arange(cols) - (cols - 1) / 2.0) * 3.0 / 600.0)
    checked = 0
    for v in range(0, n, 7):
        for c in range(cols):
            b2 = v * d_beta + np.pi + 2 * gamma[c]           # the same ray, seen from the other side
            v2 = b2 / d_beta
            if v2 > n - 1:
                continue
            i = int(np.floor(v2))
            f = v2 - i
            c2 = cols - 1 - c                                # fan angle -gamma: the mirrored column
            w2 = (1 - f) * w[i, c2] + f * w[min(i + 1, n - 1), c2]
            assert abs((w[v, c] + w2) / scale - 1.0) < 2e-2, (v, c)
            checked += 1
    assert checked > 300


def test_errors():
    with pytest.raises(ValueError, match="full turn"):
        parker_weights(circular_cone_vectors(100, 300.0, 600.0, 8, 16, 3.0).vectors, 16)
    with pytest.raises(ValueError, match="fan angle"):
        parker_weights(_short(extra=0.05), 64)


def test_plateau_views_form_one_run_in_the_middle():
    """The raw ingest folds the weight of views that are at the plateau in every column into
    the filter's output scale: those views are one run in the middle of the short scan,
    with every weight exactly the plateau value, and the rest ramp below it."""
    fan = np.arctan(0.5 * 486 * 0.299 / 680.0)
    V = 600
    g = circular_cone_vectors(V, 440.0, 680.0, 384, 486, 0.299, angular_range=(np.pi + 2 * fan) * V / (V - 1) * 1.001)
    w = parker_weights(g.vectors, 486)
    flat = np.all(w == w.max(), axis=1)
    run = np.flatnonzero(flat)
    assert len(run) > 0.6 * V and np.all(np.diff(run) == 1)
    assert run[0] > 0 and run[-1] < V - 1
    assert np.all(w[~flat].min(axis=1) < w.max())
