"""The batched bench's workload, checked on the CPU: the query plan has the stated
kind mix and selectivity range, and the bisection that sets each query's free
bound reaches its target count (measured here by brute force over the points)."""
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
import bench  # noqa: E402


def test_query_plan_mix_and_selectivities():
    kinds, sel, anchor = bench.query_plan(bench.NQ, 7)
    assert len(kinds) == len(sel) == len(anchor) == 4096
    assert np.bincount(kinds, minlength=3).tolist() == [2048, 1024, 1024]  # 50 % three, 25 % left, 25 % right
    assert sel.min() >= bench.SEL_LO and sel.max() <= bench.SEL_HI
    # log-uniform: the mean of log(sel) sits at the middle of the log range
    mid = (np.log(bench.SEL_LO) + np.log(bench.SEL_HI)) / 2
    assert abs(np.log(sel).mean() - mid) < 0.2
    assert anchor.min() >= 0 and anchor.max() < 1 << 24
    k2, s2, a2 = bench.query_plan(bench.NQ, 7)
    assert np.array_equal(kinds, k2) and np.array_equal(sel, s2) and np.array_equal(anchor, a2)


def _brute_counts(pts, kinds, min1, max1, min2):
    d1 = pts["dim1"][None, :]
    d2 = pts["dim2"][None, :]
    ok2 = d2 >= min2[:, None]
    three = (d1 >= min1[:, None]) & (d1 <= max1[:, None])
    left = d1 <= max1[:, None]
    right = d1 >= min1[:, None]
    k = kinds[:, None]
    hit = ok2 & np.where(k == 0, three, np.where(k == 1, left, right))
    return hit.sum(axis=1)


def test_calibration_reaches_targets():
    n = 1 << 16
    pts = bench.gen_points_host(n, 1)
    kinds, _, anchor = bench.query_plan(48, 3)
    # targets of 100 to 650 points: large enough that one point is within 1 %
    sel = np.exp(np.random.default_rng(4).uniform(np.log(1.5e-3), np.log(1e-2), 48))
    min1, max1, min2 = bench.calibrate(lambda k, a, b, c: _brute_counts(pts, k, a, b, c), kinds, sel, anchor, n)
    got = _brute_counts(pts, kinds, min1, max1, min2)
    err = np.abs(got - sel * n) / (sel * n)
    assert err.max() < 0.01, err  # every query within 1 % of its target count


def test_disjoint_plan_reports_every_point_once(oracle):
    """The disjoint-range workload: 4096 3-sided queries whose results partition the
    point set (every point reported by exactly one query)."""
    n = 1 << 16
    pts = bench.gen_points_host(n, 1)
    kinds, a, b, c = bench.disjoint_plan(bench.NQ, 13)
    assert (kinds == 0).all() and np.all(a[1:] > b[:-1])
    off, idx = oracle.Orc.brute_multi(pts, "f32", kinds, a, b, c)
    assert int(off[-1]) == n
    assert np.array_equal(np.sort(idx), np.arange(n, dtype=np.uint64))
    sizes = np.diff(off.astype(np.int64))
    assert sizes.max() > 100 * max(np.median(sizes), 1)  # uneven output sizes


def test_sharded_plan_routes_every_result(oracle):
    """The sharded (weak-scaling) workload on the CPU, 3 shards of 2^14 points: each
    shard's block of queries starts in its slab (right queries clipped to 3-sided
    except on the last shard), and routing by the shards' bounds loses no result:
    the routed shards' brute-force answers add up to the answer over all points."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("sh", bench.PKG_DIR / "sharded.py")
    sh = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(sh)
    world, n = 3, 1 << 14
    slabs = []
    for r in range(world):
        p = bench.gen_points_host(n, 1 + r)
        p["dim1"] += np.float32(r * bench.SLAB)
        p["dim2"] += np.float32(r * bench.SLAB)
        p["id"] += np.uint32(r * n)
        slabs.append(p)
    def counts(p, k, x, y, z):
        off, _ = oracle.Orc.brute_multi(p, "f32", k, x, y, z, counts_only=True)
        return np.diff(off.astype(np.int64))
    blocks = []
    for r in range(world):
        kinds, a, b, c, sel = bench.sharded_block(lambda k, x, y, z, s=slabs[r]: counts(s, k, x, y, z), r, world, n)
        if r < world - 1:
            assert not (kinds == 2).any()
        else:
            assert (kinds == 2).sum() == bench.NQ // 4
        three = kinds == 0
        # every 3-sided range starts in the slab (one near its top may run into the next)
        assert (a[three] >= r * bench.SLAB).all() and (a[three] < (r + 1) * bench.SLAB).all()
        blocks.append((kinds, a, b, c))
    k, a, b, c = (np.concatenate([blk[i] for blk in blocks]) for i in range(4))
    ranges = np.array([sh.shard_ranges(s) for s in slabs])
    route = sh.route_many(k, a, b, c, ranges)
    allpts = np.concatenate(slabs)
    want = counts(allpts, k, a, b, c)
    got = sum(np.where(route[:, r], counts(slabs[r], k, a, b, c), 0) for r in range(world))
    assert np.array_equal(got, want)
    # most queries stay on one shard
    assert (route.sum(axis=1) <= 1).mean() > 0.9
