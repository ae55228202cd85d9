"""CPU restatement of this build's marching cubes over active metacells -- test
infrastructure: the checker of the CUDA kernels in csrc/mc.cu, never called by the
product path.

The reference's isosurface sample (.marching-cubes/, NVIDIA's sample code behind an
OpenGL window; it does not compile in the reference's own environment, see
.marching-cubes/Notes-on-Compilation-Error.txt) is not restated: its tables are a
third party's.  This build derives its own triangle table from first principles,
and this module derives the same table the same way, independently of the C++
generator (tests compare the two tables entry for entry):

  * corner c of a cell sits at (c & 1, c >> 1 & 1, c >> 2 & 1); edge 4a + u + 2v
    runs along axis a at the other two coordinates (u, v); a corner is inside when
    its value is >= iso;
  * on each cell face the edges whose ends differ are joined in pairs: two such
    edges by one segment; four (diagonal corners inside) by two segments that each
    cut off one inside corner -- the face decides alone, so the two cells sharing
    a face agree and the surface is closed;
  * every crossed edge then has two segment ends, so the segments form loops; a
    loop is oriented so that its (Newell) normal points from the inside ends of its
    edges to the outside ends, rotated to start at its smallest edge, and fanned
    from the first vertex whose diagonals all leave the cube faces (a diagonal on a
    face would overlap the neighbouring cell).

Vertices: on the edge from global vertex a (the lower end) to b,
t = (iso - f_a) / (f_b - f_a) and the coordinate along the edge's axis is a + t, in
float32 with no fused operations; the other coordinates are a's.  A triangle is
9 float32 (three vertices x, y, z) in vertex-index units.  Output order: the given
metacells in order, their cells x fastest, then y, then z, each cell's triangles
in table order."""
from __future__ import annotations

import numpy as np

CORNERS = [((c & 1), (c >> 1) & 1, (c >> 2) & 1) for c in range(8)]


def _corner(x, y, z):
    return x | (y << 1) | (z << 2)


def _edges():
    out = []
    for a in range(3):
        o = [i for i in range(3) if i != a]
        for v in range(2):
            for u in range(2):
                lo = [0, 0, 0]
                lo[o[0]], lo[o[1]] = u, v
                hi = list(lo)
                hi[a] = 1
                out.append((_corner(*lo), _corner(*hi)))
    return out


EDGES = _edges()


def _faces():
    out = []
    for a in range(3):
        o = [i for i in range(3) if i != a]
        ring = [(0, 0), (1, 0), (1, 1), (0, 1)]
        for s in range(2):
            cs = [c for c in range(8) if CORNERS[c][a] == s]
            cs.sort(key=lambda c: ring.index((CORNERS[c][o[0]], CORNERS[c][o[1]])))
            out.append(cs)
    return out


FACES = _faces()


def _edge_between(c0, c1):
    for i, (a, b) in enumerate(EDGES):
        if {a, b} == {c0, c1}:
            return i
    raise KeyError((c0, c1))


def _faces_of_edge(e):
    a, b = EDGES[e]
    return {i for i, f in enumerate(FACES) if a in f and b in f}


def _loops(cfg):
    inside = [(cfg >> c) & 1 for c in range(8)]
    adj = {}
    for f in FACES:
        cut = [_edge_between(f[i], f[(i + 1) % 4]) for i in range(4)]
        xs = [i for i in range(4) if inside[f[i]] != inside[f[(i + 1) % 4]]]
        segs = []
        if len(xs) == 2:
            segs.append((cut[xs[0]], cut[xs[1]]))
        elif len(xs) == 4:
            segs += [(cut[(i - 1) % 4], cut[i]) for i in range(4) if inside[f[i]]]
        for a, b in segs:
            adj.setdefault(a, []).append(b)
            adj.setdefault(b, []).append(a)
    loops, seen = [], set()
    for e0 in sorted(adj):
        if e0 in seen:
            continue
        loop, prev, cur, nxt = [e0], None, e0, min(adj[e0])
        seen.add(e0)
        while nxt != e0:
            loop.append(nxt)
            seen.add(nxt)
            prev, cur = cur, nxt
            a, b = adj[cur]
            nxt = a if a != prev else b
        pts = [np.add(CORNERS[EDGES[e][0]], CORNERS[EDGES[e][1]]) for e in loop]  # twice the midpoints
        nrm = np.zeros(3, np.int64)
        for i in range(len(pts)):
            nrm += np.cross(pts[i], pts[(i + 1) % len(pts)])
        g = np.zeros(3, np.int64)
        for e in loop:
            a, b = EDGES[e]
            ins, out = (a, b) if inside[a] else (b, a)
            g += np.subtract(CORNERS[out], CORNERS[ins])
        d = int(np.dot(nrm, g))
        assert d != 0
        if d < 0:
            loop = loop[::-1]
        k = loop.index(min(loop))
        loops.append(loop[k:] + loop[:k])
    return loops


def _triangles(cfg):
    tris = []
    for loop in _loops(cfg):
        k = len(loop)
        j = next(j for j in range(k)
                 if all(not (_faces_of_edge(loop[j]) & _faces_of_edge(loop[(j + i) % k])) for i in range(2, k - 1)))
        tris += [(loop[j], loop[(j + i) % k], loop[(j + i + 1) % k]) for i in range(1, k - 1)]
    return tris


MAX_TRI = 5


def tables():
    """(ntri[256] uint8, edges[256, 15] uint8) -- the triangle table."""
    ntri = np.zeros(256, np.uint8)
    edges = np.full((256, 3 * MAX_TRI), 255, np.uint8)
    for c in range(256):
        t = _triangles(c)
        assert len(t) <= MAX_TRI
        ntri[c] = len(t)
        flat = [e for tri in t for e in tri]
        edges[c, : len(flat)] = flat
    return ntri, edges


_NTRI, _EDGES_T = tables()
_AXIS = [[i for i in range(3) if CORNERS[a][i] != CORNERS[b][i]][0] for a, b in EDGES]


def metacell_triangles(vol: np.ndarray, mc_dims, ids, iso: float) -> np.ndarray:
    """Triangles (n, 9) float32 of the cells of the given metacells, in order.
    vol: float32 (pz, py, px) vertex values."""
    pz, py, px = vol.shape
    mcx, mcy, mcz = mc_dims
    Mx = -(-(px - 1) // mcx)
    My = -(-(py - 1) // mcy)
    iso32 = np.float32(iso)
    out = []
    for mid in ids:
        mid = int(mid)
        mx, my, mz = mid % Mx, (mid // Mx) % My, mid // (Mx * My)
        x0, y0, z0 = mx * mcx, my * mcy, mz * mcz
        x1, y1, z1 = min(x0 + mcx, px - 1), min(y0 + mcy, py - 1), min(z0 + mcz, pz - 1)
        for z in range(z0, z1):
            for y in range(y0, y1):
                for x in range(x0, x1):
                    f = [vol[z + cz, y + cy, x + cx] for cx, cy, cz in CORNERS]
                    cfg = sum(1 << c for c in range(8) if f[c] >= iso32)
                    n = int(_NTRI[cfg])
                    for k in range(n):
                        tri = []
                        for e in _EDGES_T[cfg, 3 * k: 3 * k + 3]:
                            a, b = EDGES[e]
                            t = np.float32((iso32 - f[a]) / np.float32(f[b] - f[a]))
                            p = [np.float32(x + CORNERS[a][0]), np.float32(y + CORNERS[a][1]),
                                 np.float32(z + CORNERS[a][2])]
                            p[_AXIS[e]] = np.float32(p[_AXIS[e]] + t)
                            tri += p
                        out.append(tri)
    return np.asarray(out, np.float32).reshape(-1, 9)


def mesh_defects(tri: np.ndarray, dims) -> tuple[int, int]:
    """(directed edges used twice, interior edges without their reverse) of a
    triangle soup, vertices matched by their bits; boundary edges (both ends on
    the volume's outer faces) may be unmatched."""
    px, py, pz = dims
    v = np.ascontiguousarray(tri.reshape(-1, 3)).view(np.uint32).reshape(-1, 3)
    keys = [tuple(r) for r in v.tolist()]
    from collections import Counter
    de = Counter()
    for i in range(0, len(keys), 3):
        for j in range(3):
            de[(keys[i + j], keys[i + (j + 1) % 3])] += 1
    dup = sum(1 for c in de.values() if c != 1)
    lim = np.array([px - 1, py - 1, pz - 1], np.float32)

    def on_boundary(k):
        p = np.array(k, np.uint32).view(np.float32)
        return bool(np.any(p == 0) or np.any(p == lim))
    open_ = sum(1 for (a, b) in de if (b, a) not in de and not (on_boundary(a) and on_boundary(b)))
    return dup, open_
