"""The oracle's many-query brute force (orc_brute_multi, used to check the large
configurations) equals its one-query brute force, query by query, for every value
type, with ties, unordered ids and any thread count."""
import numpy as np
import pytest

from datagen import rand_points, rand_queries


@pytest.mark.parametrize("dt", ["f32", "f64", "i32"])
@pytest.mark.parametrize("threads", [1, 3, 16])
def test_brute_multi_equals_brute(oracle, dt, threads):
    pts = rand_points(20011, dt, ids="random", dup=(threads == 3), seed=41)
    qs = rand_queries(pts, 40, seed=42) + [("three", 5, 1, 0), ("left", 0, -10**9, 0), ("right", 10**9, 0, 0)]
    kinds = [oracle.KINDS[q[0]] for q in qs]
    col = lambda j: [q[j] for q in qs]  # noqa: E731
    off, idx = oracle.Orc.brute_multi(pts, dt, kinds, col(1), col(2), col(3), threads=threads)
    assert len(off) == len(qs) + 1 and off[-1] == len(idx)
    for i, q in enumerate(qs):
        want = oracle.Orc.brute(pts, dt, *q)
        assert np.array_equal(idx[off[i]:off[i + 1]], want), (i, q)


def test_brute_multi_empty(oracle):
    pts = rand_points(0, "f32")
    off, idx = oracle.Orc.brute_multi(pts, "f32", [0, 1], [0, 0], [1, 1], [0, 0])
    assert off.tolist() == [0, 0, 0] and len(idx) == 0
