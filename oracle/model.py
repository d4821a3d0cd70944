"""TEST INFRASTRUCTURE ONLY: CPU restatement of minirecast model.py:18-29 (otsu_threshold).

The GPU path must return the reference's threshold bit for bit, so this restatement keeps
numpy's primitives and the reference's order of FP64 operations: the non-zero voxels, their
0.1 / 99.95 percentiles (numpy "linear"), a histogram of the values clipped to that range,
then the bin centre that maximises the between-class variance w0 * w1 * (m0 - m1)^2 with
w0 / m0 the weight and mean of the bins up to and including a centre, w1 / m1 those above
it. Pinned against the reference's own output in tests/golden/misc.npz.
"""
import numpy as np


def otsu_threshold(vol, bins=512):
    """model.py:18-29."""
    vals = np.asarray(vol)
    vals = vals[vals != 0]                                        # model.py:20
    lo, hi = np.percentile(vals, [0.1, 99.95])                    # model.py:21
    counts, edges = np.histogram(np.clip(vals, lo, hi), bins=bins, range=(lo, hi))
    mid = 0.5 * (edges[1:] + edges[:-1])                          # model.py:23
    below = np.cumsum(counts)                                     # weight up to each bin
    above = below[-1] - below
    moment = np.cumsum(counts * mid)
    mean_below = moment / np.maximum(below, 1)
    mean_above = (np.sum(counts * mid) - moment) / np.maximum(above, 1)
    between = below * above * (mean_below - mean_above) ** 2     # model.py:28
    return float(mid[int(np.argmax(between))])
