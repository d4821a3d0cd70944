"""TEST INFRASTRUCTURE ONLY: the marching-cubes case table, generated in Python from the
cube's geometry, to check the table that the CUDA library builds on its own (csrc/surface.cu)
and to drive the CPU marching-cubes oracle (oracle/model.py).

Cube corners c = dx + 2 dy + 4 dz (dx along the volume's first axis). Edges are numbered
axis by axis: edges 0-3 run along axis 0 from the corners with dx = 0 (in corner order),
4-7 along axis 1, 8-11 along axis 2. A corner is inside when its value is above the iso
level; an edge with one inside and one outside corner carries one surface vertex.

For each of the 256 inside/outside patterns the surface inside the cube is built face by
face: on every cube face, walked counter-clockwise as seen from outside, each edge where
the walk leaves the inside region ("exit") is joined to the edge where that run of inside
corners was entered ("entry"). On a face whose inside corners are diagonal opposites (the
ambiguous face) every inside corner is cut off on its own. The rule depends only on the
face's four corners, so the two cubes sharing a face cut it the same way and the surface
is closed across cubes. Joining the face segments edge to edge gives closed loops, each
fanned into triangles from the first vertex whose diagonals stay off the cube faces,
oriented so that the triangle normal (right-hand rule) points from the inside corners to
the outside ones. At most 5 triangles per cube.
"""
import numpy as np

MAX_TRIANGLES = 5


def _geometry():
    P = np.array([[c & 1, (c >> 1) & 1, (c >> 2) & 1] for c in range(8)], float)
    edges = [(c0, c0 | (1 << a)) for a in range(3) for c0 in range(8) if not (c0 >> a) & 1]
    index = {frozenset(e): i for i, e in enumerate(edges)}
    faces = []
    for a in range(3):
        for side in (0, 1):
            cs = [c for c in range(8) if ((c >> a) & 1) == side]
            normal = np.zeros(3)
            normal[a] = 1.0 if side else -1.0
            centre = P[cs].mean(0)
            u = np.zeros(3)
            u[(a + 1) % 3] = 1.0
            v = np.cross(normal, u)
            angle = [np.arctan2((P[c] - centre) @ v, (P[c] - centre) @ u) for c in cs]
            faces.append([c for _, c in sorted(zip(angle, cs))])     # counter-clockwise from outside
    return P, edges, index, faces


def _loops(mask, index, faces):
    inside = [(mask >> c) & 1 for c in range(8)]
    nxt = {}
    for cs in faces:
        ambiguous = sum(inside[c] for c in cs) == 2 and inside[cs[0]] == inside[cs[2]]
        for i in range(4):
            q, qn = cs[i], cs[(i + 1) % 4]
            if not (inside[q] and not inside[qn]):
                continue                                    # not an exit
            j = i
            if not ambiguous:
                while inside[cs[(j - 1) % 4]]:
                    j = (j - 1) % 4
            entry = index[frozenset((cs[(j - 1) % 4], cs[j]))]
            nxt[index[frozenset((q, qn))]] = entry
    loops, seen = [], set()
    for e0 in sorted(nxt):
        if e0 in seen:
            continue
        loop, e = [e0], nxt[e0]
        seen.add(e0)
        while e != e0:
            loop.append(e)
            seen.add(e)
            e = nxt[e]
        loops.append(loop)
    return loops


def _share_face(e1, e2, edges, faces):
    corners = set(edges[e1]) | set(edges[e2])
    return any(corners <= set(f) for f in faces)


def build():
    """(triangles int8 [256, 15]: three edge numbers per triangle, -1 after the last;
    counts int32 [256])."""
    P, edges, index, faces = _geometry()
    tri = -np.ones((256, 3 * MAX_TRIANGLES), np.int8)
    cnt = np.zeros(256, np.int32)
    for m in range(256):
        out = []
        for loop in _loops(m, index, faces):
            # the face walks give every loop the same turning sense: its normal points
            # into the inside corners; reversed, it points out of them
            loop = loop[::-1]
            # fan from the first vertex none of whose diagonals lies on a cube face (such a
            # diagonal would touch the neighbouring cell's surface along that face)
            n = len(loop)
            for r in range(n):
                if not any(_share_face(loop[r], loop[(r + i) % n], edges, faces) for i in range(2, n - 1)):
                    break
            loop = loop[r:] + loop[:r]
            out.extend((loop[0], loop[i], loop[i + 1]) for i in range(1, len(loop) - 1))
        assert len(out) <= MAX_TRIANGLES
        cnt[m] = len(out)
        for i, t in enumerate(out):
            tri[m, 3 * i:3 * i + 3] = t
    return tri, cnt


EDGES = _geometry()[1]          # (corner a, corner b) of each edge, b = a + 2^axis
TRIANGLES, COUNTS = build()
