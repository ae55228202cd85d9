"""Whole blocks: queries whose min2 lies below entire subtrees, so the search
reports those subtrees from the per-block subtree minimum (TreeDev::sub_min)
without testing their dim2.  Every result set must still equal the oracle's,
including trees with low outliers below such blocks (which must stop the
shortcut there), signed zeros, ties, a sparse last level, and trees read back
from an image (whose index is rebuilt on load)."""
import numpy as np
import pytest

from datagen import rand_points

pytestmark = pytest.mark.gpu


def _oracle_set(oracle, ref, kind, a, b, m2, points):
    if points:
        return oracle.canon(oracle.Orc.search_points(ref, kind, a, b, m2))
    return oracle.canon(oracle.Orc.search_ids(ref, kind, a, b, m2))


def _low_min2_queries(pts, k, seed):
    """Mixed kinds whose min2 sits at or below the dim1 range (so every subtree
    inside the range qualifies whole), plus a few with min2 inside the data."""
    rng = np.random.default_rng(seed)
    d1 = np.sort(pts["dim1"])
    d2 = pts["dim2"]
    out = []
    for i in range(k):
        kind = ["three", "left", "right"][i % 3]
        a, b = sorted(rng.choice(d1, 2))
        if i % 4 == 3:
            m2 = rng.choice(d2)
        elif kind == "three":
            m2 = a
        elif kind == "left":
            m2 = d1[0]
        else:
            m2 = a
        out.append((kind, a, b, m2))
    return out


@pytest.mark.parametrize("dt", ["f32", "f64", "i32"])
@pytest.mark.parametrize("n,ids", [(300001, "arange"), (131072, "random"), (70000, "none")])
def test_whole_blocks_single(pst, oracle, dt, n, ids):
    pts = rand_points(n, dt, ids=ids, seed=n + 3, width=5.0, signed_zero=(dt != "i32"))
    ref = oracle.Orc.build(pts, dt)
    tr = pst.StaticPSTGPU.from_numpy(pts, dt)
    for i, (kind, a, b, m2) in enumerate(_low_min2_queries(pts, 18, seed=n)):
        points = (i % 2 == 1) or ids == "none"
        got = tr.search(kind, a, b, m2, ret="points" if points else "ids")
        assert np.array_equal(oracle.canon(got), _oracle_set(oracle, ref, kind, a, b, m2, points)), (kind, a, b, m2)
        assert tr.count(kind, a, b, m2) == len(got)
    tr.close()


@pytest.mark.parametrize("dt", ["f32", "f64", "i32"])
def test_whole_blocks_batched(pst, oracle, dt):
    pts = rand_points(400000, dt, ids="random", seed=77, width=3.0)
    ref = oracle.Orc.build(pts, dt)
    tr = pst.StaticPSTGPU.from_numpy(pts, dt)
    qs = _low_min2_queries(pts, 96, seed=78)
    q = pst.make_queries([pst.pst.KIND[k] for k, *_ in qs], [x[1] for x in qs], [x[2] for x in qs],
                         [x[3] for x in qs], dt)
    eng = pst.BatchEngine(tr, max_queries=128)
    offs, res = eng.search(q)
    for i, (kind, a, b, m2) in enumerate(qs):
        assert np.array_equal(oracle.canon(res[offs[i]:offs[i + 1]]),
                              _oracle_set(oracle, ref, kind, a, b, m2, False)), i
    offs2, res2 = eng.search(q, ret="points")
    for i in range(0, len(qs), 5):
        kind, a, b, m2 = qs[i]
        assert np.array_equal(oracle.canon(res2[offs2[i]:offs2[i + 1]]),
                              _oracle_set(oracle, ref, kind, a, b, m2, True)), i
    eng.close()
    tr.close()


@pytest.mark.parametrize("dt", ["f32", "f64", "i32"])
def test_whole_blocks_low_outliers(pst, oracle, dt):
    """Scattered points whose dim2 lies far below every query's min2 sink to the
    bottom of the tree: the blocks above them must not be taken whole (their
    subtree minimum is below min2), their neighbours still are, and the reported
    sets stay the oracle's."""
    pts = rand_points(200000, dt, ids="arange", seed=5, lo=1000.0, hi=2000.0, width=2.0)
    rng = np.random.default_rng(6)
    low = rng.choice(len(pts), 400, replace=False)
    pts["dim2"][low] = pts["dim2"][low] - pts["dim2"].dtype.type(1500)
    ref = oracle.Orc.build(pts, dt)
    tr = pst.StaticPSTGPU.from_numpy(pts, dt)
    for kind, a, b, m2 in _low_min2_queries(pts, 24, seed=7):
        got = tr.search(kind, a, b, m2, ret="ids")
        assert np.array_equal(oracle.canon(got), _oracle_set(oracle, ref, kind, a, b, m2, False)), (kind, a, b, m2)
    tr.close()


def test_whole_blocks_after_image(pst, oracle):
    """A tree read back from its image rebuilds the subtree minima and answers
    whole-block queries like the original."""
    pts = rand_points(150000, "f32", ids="random", seed=9, width=4.0)
    ref = oracle.Orc.build(pts, "f32")
    tr = pst.StaticPSTGPU.from_numpy(pts, "f32")
    back = pst.StaticPSTGPU.from_bytes(tr.to_bytes())
    tr.close()
    for kind, a, b, m2 in _low_min2_queries(pts, 12, seed=10):
        got = back.search(kind, a, b, m2, ret="ids")
        assert np.array_equal(oracle.canon(got), _oracle_set(oracle, ref, kind, a, b, m2, False)), (kind, a, b, m2)
    back.close()


@pytest.mark.parametrize("dt", ["f32", "f64", "i32"])
@pytest.mark.parametrize("n", [127, 128, 200, 255, 256, 511, 1000])
def test_whole_blocks_smallest_trees(pst, oracle, dt, n):
    """Trees of 7 to 10 levels: the subtree minima exist from 8 levels on (one
    64-slot block level at first), below that the shortcut is off.  Every query
    of the whole-block mix, plus the extremes, against the oracle."""
    pts = rand_points(n, dt, ids="random", seed=n + 17, width=3.0)
    ref = oracle.Orc.build(pts, dt)
    tr = pst.StaticPSTGPU.from_numpy(pts, dt)
    qs = _low_min2_queries(pts, 12, seed=n)
    lo, hi = (-(2 ** 31), 2 ** 31 - 1) if dt == "i32" else (-np.inf, np.inf)
    qs += [("three", lo, hi, lo), ("left", 0, hi, lo), ("right", lo, 0, lo)]
    for kind, a, b, m2 in qs:
        got = tr.search(kind, a, b, m2, ret="ids")
        assert np.array_equal(oracle.canon(got), _oracle_set(oracle, ref, kind, a, b, m2, False)), (kind, a, b, m2)
    tr.close()
