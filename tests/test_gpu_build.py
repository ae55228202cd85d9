"""GPU construction parity: the exported tree equals the oracle's tree bit for bit
(every field of every slot, in the reference's layout)."""
import numpy as np
import pytest

from datagen import rand_points

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 3, 4, 5, 7, 8, 9, 31, 32, 33, 63, 64, 65, 100, 1000, 2047, 2048, 2049, 4095, 4096, 4097,
         10000, 65537, 300001]


def _compare(pst, oracle, pts, dt):
    ref = oracle.Orc.build(pts, dt)
    tr = pst.StaticPSTGPU.from_numpy(pts, dt)
    ex = tr.export()
    assert tr.info()["slots"] == ref.S
    for f in ("dim1", "dim2", "med", "bitcodes"):
        a, b = ex[f], getattr(ref, f)
        ua, ub = a.view(f"u{a.itemsize}"), b.view(f"u{b.itemsize}")
        bad = np.nonzero(ua != ub)[0]
        assert len(bad) == 0, f"{f} differs (n={len(pts)}, first slots {bad[:5]})"
    if ref.has_id:
        assert ex["ids"].tobytes() == ref.ids.tobytes(), "ids differ"
    tr.close()


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("dt", ["f32", "f64", "i32"])
def test_tree_matches_oracle(pst, oracle, n, dt):
    _compare(pst, oracle, rand_points(n, dt, ids="arange", seed=n), dt)


@pytest.mark.parametrize("ids", ["random", "desc", "const", "none"])
@pytest.mark.parametrize("n", [1, 17, 1000, 5000, 70001])
@pytest.mark.parametrize("dt", ["f32", "f64", "i32"])
def test_tree_ids_and_ties(pst, oracle, n, dt, ids):
    """Heavy value ties and every id pattern: the (value, id, index) order decides."""
    _compare(pst, oracle, rand_points(n, dt, ids=ids, dup=True, seed=3 * n + 1), dt)


@pytest.mark.parametrize("dt", ["f32", "f64"])
def test_tree_signed_zero(pst, oracle, dt):
    """-0.0 and +0.0 compare equal in the reference's comparators."""
    _compare(pst, oracle, rand_points(20000, dt, ids="random", signed_zero=True, lo=-5, hi=5, seed=9), dt)


def test_tree_all_equal(pst, oracle):
    pts = rand_points(5000, "f32", ids="random", seed=4)
    pts["dim1"] = 3.0
    pts["dim2"] = 3.0
    _compare(pst, oracle, pts, "f32")


def test_empty_tree(pst):
    pts = rand_points(0, "f32")
    tr = pst.StaticPSTGPU.from_numpy(pts, "f32")
    assert tr.info()["levels"] == 0
    assert len(tr.search("three", 0, 10, 0)) == 0
    assert len(tr.twoSidedLeftSearch(5, 0, ret="ids")) == 0
