"""Pins the oracle (the C restatement) to the reference itself: StaticPSTCPUIter
compiled unmodified from its sources into oracle/_ref/.  Whole trees must be
identical bit for bit, and every search must return the same multiset."""
import numpy as np
import pytest

from datagen import rand_points, rand_queries


def _ref_available(oracle):
    if not oracle.Ref.available():
        pytest.skip("oracle/_ref/libpstref.so not built (reference sources absent)")


CASES = [(n, dt, ids, dup) for dt in ("f32", "f64", "i32") for ids in ("arange", "random", "desc", "none")
         for n, dup in ((0, False), (1, False), (2, True), (3, True), (7, True), (8, False), (33, True),
                        (100, False), (1000, True), (4097, False))]


@pytest.mark.parametrize("n,dt,ids,dup", CASES)
def test_tree_and_searches_match_reference(oracle, n, dt, ids, dup):
    _ref_available(oracle)
    pts = rand_points(n, dt, ids=ids, dup=dup, seed=1000 + n)
    mine = oracle.Orc.build(pts, dt)
    ref = oracle.Ref(pts, dt)
    assert mine.equal(ref.export())
    for kind, a, b, m2 in rand_queries(pts, 10, seed=n):
        want = ref.search(kind, a, b, m2, points=True)
        got = oracle.Orc.search_points(mine, kind, a, b, m2)
        assert np.array_equal(oracle.canon(got), oracle.canon(want))
        if ids != "none":
            assert np.array_equal(oracle.canon(oracle.Orc.search_ids(mine, kind, a, b, m2)),
                                  oracle.canon(ref.search(kind, a, b, m2)))
        assert len(oracle.Orc.brute(pts, dt, kind, a, b, m2)) == len(want)
    ref.close()


def test_signed_zero_matches_reference(oracle):
    _ref_available(oracle)
    pts = rand_points(3000, "f32", ids="random", signed_zero=True, lo=-3, hi=3, seed=5)
    assert oracle.Orc.build(pts, "f32").equal(oracle.Ref(pts, "f32").export())


def test_config1_counts(oracle):
    """2^20 points, dim1 ~ U[0,1000), dim2 = dim1 + U[0,50): reference and oracle
    agree on the 3-sided (400, 420, 430) and 2-sided-left (500, 500) results."""
    _ref_available(oracle)
    rng = np.random.default_rng(1)
    n = 1 << 20
    d1 = (rng.random(n, dtype=np.float32) * np.float32(1000)).astype(np.float32)
    d2 = (d1 + rng.random(n, dtype=np.float32) * np.float32(50)).astype(np.float32)
    pts = oracle.make_points(d1, d2, np.arange(n, dtype=np.uint32), "f32")
    mine = oracle.Orc.build(pts, "f32")
    ref = oracle.Ref(pts, "f32")
    assert mine.equal(ref.export())
    for kind, a, b, m2 in (("three", 400, 420, 430), ("left", 0, 500, 500)):
        assert np.array_equal(oracle.canon(oracle.Orc.search_ids(mine, kind, a, b, m2)),
                              oracle.canon(ref.search(kind, a, b, m2)))
