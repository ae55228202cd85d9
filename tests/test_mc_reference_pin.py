"""The marching-cubes triangle table against the reference's isosurface sample
(.marching-cubes/marchingCubes_kernel.cu:155-413 with .marching-cubes/tables.h),
through tests/golden/mc_reference_cases.npz, which tests/golden/make_mc_fixture.py
derives from those files.

The two tables number corners and edges differently and use opposite bits (the
sample sets bit i when corner i is below the isovalue; this library when corner i
is at or above it), so every case is compared through the geometry: for each of the
256 inside/outside patterns of a cell's corners, the set of cell edges the sample's
triangles put vertices on equals the set this library's triangles use, and both
equal the edges whose two corners differ.  The surface therefore passes through
the same edge points in every cell (the interpolated point on an edge depends on
the edge's two values only).  Triangle counts agree except on the cases where a
face or the cell interior is ambiguous, which each table resolves its own way; the
library's choice closes the surface across faces (tests/test_mc_cpu.py)."""
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import marching_cubes as mc  # noqa: E402

FIX = Path(__file__).resolve().parent / "golden" / "mc_reference_cases.npz"


def _geo_edge(c0, c1, corners):
    return frozenset((tuple(corners[c0]), tuple(corners[c1])))


def _compare():
    d = np.load(FIX)
    ref_corners = [tuple(int(v) for v in c) for c in d["corners"]]
    ref_edges = [_geo_edge(a, b, ref_corners) for a, b in d["edge_corners"]]
    my_corners = [tuple(c) for c in mc.CORNERS]
    my_edges = [_geo_edge(a, b, my_corners) for a, b in mc.EDGES]
    ntri, edges = mc.tables()
    differ = []
    for case in range(256):
        below = {ref_corners[i] for i in range(8) if (case >> int(d["below_bit"][i])) & 1}
        my_case = sum(1 << j for j, c in enumerate(my_corners) if c not in below)  # at or above: inside
        ref_set = {ref_edges[e] for e in range(12) if (int(d["tri_edge_mask"][case]) >> e) & 1}
        my_set = {my_edges[int(e)] for e in edges[my_case, :3 * int(ntri[my_case])]}
        crossed = {e for e in ref_edges if len({p in below for p in e}) == 2}
        assert ref_set == crossed, case
        assert my_set == crossed, case
        assert ({ref_edges[e] for e in range(12) if (int(d["edge_table"][case]) >> e) & 1}) == crossed
        if int(d["num_verts"][case]) != 3 * int(ntri[my_case]):
            differ.append(case)
    return differ


def test_same_crossed_edges_as_the_reference_sample():
    differ = _compare()
    # the cases whose triangle counts differ all have an ambiguous face: two
    # diagonal corners inside and the other two outside on one face
    d = np.load(FIX)
    corners = [tuple(int(v) for v in c) for c in d["corners"]]
    faces = []
    for axis in range(3):
        for side in (0, 1):
            faces.append([i for i, c in enumerate(corners) if c[axis] == side])
    for case in differ:
        below = [(case >> int(d["below_bit"][i])) & 1 for i in range(8)]
        amb = False
        for f in faces:
            pts = sorted(f, key=lambda i: [corners[i][a] for a in range(3)])
            # a face's corners ordered so that 0-3 and 1-2 are its diagonals
            a, b, c, e = pts
            if below[a] == below[e] and below[b] == below[c] and below[a] != below[b]:
                amb = True
        assert amb, case
    assert len(differ) < 256
