"""The library's marching-cubes triangle table (generated by the C++ library at
load) equals the one the CPU restatement derives independently; and the table
gives closed, consistently oriented surfaces (checked on the CPU restatement)."""
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import marching_cubes as mc  # noqa: E402


def test_tables_match_cpu_restatement(pst):
    ntri, edges = pst.marchingCubesTables()
    want_n, want_e = mc.tables()
    assert np.array_equal(ntri, want_n)
    for c in range(256):
        k = 3 * int(want_n[c])
        assert np.array_equal(edges[c, :k], want_e[c, :k]), c
    assert int(ntri.max()) == 5 and int(ntri[0]) == 0 and int(ntri[255]) == 0


def test_surface_is_closed_and_oriented():
    rng = np.random.default_rng(7)
    for shape in ((9, 10, 11), (6, 13, 7)):
        vol = rng.random(shape).astype(np.float32)
        pz, py, px = shape
        M = [-(-(d - 1) // 3) for d in (px, py, pz)]
        tri = mc.metacell_triangles(vol, (3, 3, 3), range(M[0] * M[1] * M[2]), 0.5)
        assert len(tri) > 0
        assert mc.mesh_defects(tri, (px, py, pz)) == (0, 0)
