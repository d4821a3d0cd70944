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


def marching_cubes(vol, iso, origin=(0.0, 0.0, 0.0), spacing=1.0):
    """CPU marching cubes with the case table of oracle/mc_table.py, in the device path's
    FP32 arithmetic and output order: (points [V, 3] float32 in grid-edge order, faces [F, 3])."""
    from .mc_table import TRIANGLES, COUNTS, EDGES
    v = np.ascontiguousarray(vol, dtype=np.float32)
    nx, ny, nz = v.shape
    iso = np.float32(iso)
    corner = []
    for c in range(8):
        dx, dy, dz = c & 1, (c >> 1) & 1, (c >> 2) & 1
        corner.append(v[dx:nx - 1 + dx, dy:ny - 1 + dy, dz:nz - 1 + dz].reshape(-1))
    case = np.zeros(corner[0].shape, np.int64)
    for c in range(8):
        case |= (corner[c] > iso).astype(np.int64) << c
    cell = np.arange(case.size)
    ci, rest = np.divmod(cell, (ny - 1) * (nz - 1))
    cj, ck = np.divmod(rest, nz - 1)
    cnt = COUNTS[case]
    rows = []
    for t in range(5):
        sel = np.nonzero(cnt > t)[0]
        for q in range(3):
            e = TRIANGLES[case[sel], 3 * t + q].astype(np.int64)
            a = np.array([EDGES[x][0] for x in range(12)])[e]
            b = np.array([EDGES[x][1] for x in range(12)])[e]
            axis = np.where(b - a == 1, 0, np.where(b - a == 2, 1, 2))
            ia, ja, ka = ci[sel] + (a & 1), cj[sel] + ((a >> 1) & 1), ck[sel] + ((a >> 2) & 1)
            va = np.choose(a, [corner[c][sel] for c in range(8)])
            vb = np.choose(b, [corner[c][sel] for c in range(8)])
            s = (iso - va) / (vb - va)                       # float32
            coord = [ia.astype(np.float32), ja.astype(np.float32), ka.astype(np.float32)]
            for ax in range(3):
                coord[ax] = np.where(axis == ax, coord[ax] + s, coord[ax]).astype(np.float32)
            pos = np.stack([np.float32(origin[ax]) + np.float32(spacing) * coord[ax] for ax in range(3)], 1)
            eid = ((ia * ny + ja) * nz + ka) * 3 + axis
            rows.append((sel, t, q, eid, pos))
    if not rows or sum(len(r[0]) for r in rows) == 0:
        return np.zeros((0, 3), np.float32), np.zeros((0, 3), np.int64)
    sel = np.concatenate([r[0] for r in rows])
    tq = np.concatenate([np.full(len(r[0]), 3 * r[1] + r[2]) for r in rows])
    eid = np.concatenate([r[3] for r in rows])
    pos = np.concatenate([r[4] for r in rows]).astype(np.float32)
    order = np.lexsort((tq, sel))                             # cell order, then slot
    eid, pos = eid[order], pos[order]
    uniq, first, inv = np.unique(eid, return_index=True, return_inverse=True)
    return pos[first], inv.reshape(-1, 3)
