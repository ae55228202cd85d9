"""Serving loop: results in the mix equal the same queries run alone; continuous
batching across several resident trees; admission under a small result arena;
cancellation and bounded waits."""
import time

import numpy as np
import pytest

from datagen import rand_points, rand_queries

pytestmark = pytest.mark.gpu


def _queries(pst, qs, dt):
    return pst.make_queries([pst.pst.KIND[k] for k, *_ in qs], [x[1] for x in qs], [x[2] for x in qs],
                            [x[3] for x in qs], dt)


@pytest.mark.parametrize("slots", [1, 3])
def test_mix_equals_alone(pst, oracle, slots):
    trees, qsets = [], []
    specs = [(30000, "f32", 1), (120000, "f64", 2), (5000, "i32", 3), (250000, "f32", 4)]
    for n, dt, seed in specs:
        pts = rand_points(n, dt, ids="random", dup=(dt == "i32"), seed=seed)
        trees.append((pst.StaticPSTGPU.from_numpy(pts, dt), dt))
        qsets.append(rand_queries(pts, 60, seed=seed + 10))
    srv = pst.Server(max_batch=16, slots_per_tree=slots, out_budget_bytes=64 << 20)
    idx = [srv.add_tree(t) for t, _ in trees]
    # interleave submissions of all trees in small bursts so batches form while others run
    sub = []
    for j in range(0, 60, 5):
        for ti, (t, dt) in enumerate(trees):
            q = _queries(pst, qsets[ti][j:j + 5], dt)
            ids = srv.submit(idx[ti], q, ret="ids")
            sub += [(ti, j + k, int(r)) for k, r in enumerate(ids)]
    srv.drain(120000)
    for ti, qi, rid in sub:
        t, dt = trees[ti]
        kind, a, b, m2 = qsets[ti][qi]
        got = srv.take(rid, np.uint32)
        alone = t.search(kind, a, b, m2, ret="ids")
        assert np.array_equal(np.sort(got), np.sort(alone)), (ti, qi)
    st = srv.stats()
    assert st["completed"] == len(sub) and st["failed"] == 0
    assert st["batches"] >= len(sub) // 16
    assert st["p99_ms"] >= st["p50_ms"] > 0
    srv.close()
    for t, _ in trees:
        t.close()


def test_points_and_admission(pst):
    """A 1 MiB result arena forces batches to wait for memory (and an oversized
    request to fail alone) while the rest complete correctly."""
    pts = rand_points(200000, "f32", ids="arange", seed=9)
    t = pst.StaticPSTGPU.from_numpy(pts, "f32")
    srv = pst.Server(max_batch=8, slots_per_tree=2, out_budget_bytes=1 << 20)
    i = srv.add_tree(t)
    qs = [("left", 0, 50 + 10 * k, 55 + 10 * k) for k in range(20)]
    qs.append(("three", -1, 2000, -1))  # every point: 2.4 MB of records > 1 MiB arena
    ids = srv.submit(i, _queries(pst, qs, "f32"), ret="points")
    srv.drain(60000)
    rec = pst.point_dtype("f32", True)
    for k, rid in enumerate(ids[:-1]):
        got = srv.take(rid, rec)
        alone = t.search(*qs[k], ret="points")
        assert np.array_equal(np.sort(got["id"]), np.sort(alone["id"]))
    st, cnt = srv.wait(ids[-1])
    assert st == 3 and cnt == len(pts)  # PST_ERR_NOMEM
    assert srv.stats()["peak_out_bytes"] <= 1 << 20
    srv.close()
    t.close()


def test_cancel_and_timeout(pst):
    pts = rand_points(100000, "f32", seed=5)
    t = pst.StaticPSTGPU.from_numpy(pts, "f32")
    srv = pst.Server(max_batch=4, slots_per_tree=1)
    i = srv.add_tree(t)
    q = _queries(pst, [("left", 0, 500, 500)] * 40, "f32")
    ids = srv.submit(i, q)
    srv.cancel(ids[-1])
    try:
        srv.wait(ids[-2], timeout_ms=0)
    except pst.PSTError as e:
        assert e.status == 8  # PST_ERR_TIMEOUT while still queued
    srv.drain(60000)
    assert srv.stats()["cancelled"] + srv.stats()["completed"] == 40
    with pytest.raises(pst.PSTError):
        srv.submit(7, q[:1])  # unknown tree
    srv.close()
    t.close()


def test_open_loop_latency(pst):
    """Poisson arrivals: latency is measured from the scheduled arrival."""
    pts = rand_points(1 << 20, "f32", seed=2)
    t = pst.StaticPSTGPU.from_numpy(pts, "f32")
    srv = pst.Server(max_batch=256, slots_per_tree=2, keep_results=False)
    i = srv.add_tree(t)
    rng = np.random.default_rng(1)
    n = 2000
    gaps = rng.exponential(1 / 20000.0, n)
    iso = rng.uniform(0, 1000, n).astype(np.float32)
    q = pst.make_queries(np.ones(n, np.int32), np.zeros(n), iso, iso, "f32")
    t0 = time.monotonic_ns()
    arrive = t0 + np.cumsum(gaps * 1e9).astype(np.uint64)
    k = 0
    while k < n:
        now = time.monotonic_ns()
        j = int(np.searchsorted(arrive, now, side="right"))
        if j > k:
            srv.submit(i, q[k:j], arrival_ns=arrive[k:j])
            k = j
    srv.drain(60000)
    st = srv.stats()
    assert st["completed"] == n and 0 < st["p50_ms"] <= st["p99_ms"] < 1000
    srv.close()
    t.close()


def test_admission_into_free_hbm(pst, oracle):
    """With a headroom set, batches whose results do not fit a 1 MiB arena (one
    request alone needs 2.4 MB) are admitted into free HBM, one batch at a time,
    instead of failing; every result equals the oracle's."""
    pts = rand_points(200000, "f32", ids="arange", seed=19)
    ref = oracle.Orc.build(pts, "f32")
    t = pst.StaticPSTGPU.from_numpy(pts, "f32")
    srv = pst.Server(max_batch=8, slots_per_tree=2, out_budget_bytes=1 << 20, keep_results=1,
                     hbm_headroom_bytes=1 << 30)
    i = srv.add_tree(t)
    qs = [("left", 0, 50 + 40 * k, 55 + 40 * k) for k in range(24)] + [("three", -1, 2000, -1)] * 3
    ids = srv.submit(i, _queries(pst, qs, "f32"), ret="points")
    srv.drain(60000)
    for (kind, a, b, m2), rid in zip(qs, ids):
        got = srv.take(int(rid), pts.dtype)
        want = oracle.Orc.search_points(ref, kind, a, b, m2)
        assert np.array_equal(oracle.canon(got), oracle.canon(want)), (kind, a, b, m2)
    st = srv.stats()
    assert st["failed"] == 0 and st["completed"] == len(qs)
    assert st["spilled"] >= 1  # the whole-tree requests (batched together or not) went past the arena
    srv.close()
    t.close()
