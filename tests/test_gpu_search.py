"""GPU search parity: every query's result set equals the oracle's (ids or whole
points, compared as sorted multisets, bit-exact)."""
import numpy as np
import pytest

from datagen import rand_points, rand_queries

pytestmark = pytest.mark.gpu


def _oracle_set(oracle, tree, kind, a, b, m2, points):
    if points or not tree.has_id:
        return oracle.canon(oracle.Orc.search_points(tree, kind, a, b, m2))
    return oracle.canon(oracle.Orc.search_ids(tree, kind, a, b, m2))


@pytest.mark.parametrize("dt", ["f32", "f64", "i32"])
@pytest.mark.parametrize("n,ids,dup", [(1, "arange", False), (2, "arange", False), (33, "random", True),
                                       (1000, "arange", False), (4097, "random", True), (50000, "desc", False),
                                       (50000, "none", True), (200003, "arange", False)])
def test_plain_search(pst, oracle, dt, n, ids, dup):
    pts = rand_points(n, dt, ids=ids, dup=dup, seed=n + 5)
    ref = oracle.Orc.build(pts, dt)
    tr = pst.StaticPSTGPU.from_numpy(pts, dt)
    for i, (kind, a, b, m2) in enumerate(rand_queries(pts, 12, seed=n)):
        points = (i % 2 == 1) or ids == "none"
        got = tr.search(kind, a, b, m2, ret="points" if points else "ids")
        assert np.array_equal(oracle.canon(got), _oracle_set(oracle, ref, kind, a, b, m2, points)), (kind, a, b, m2)
        assert tr.count(kind, a, b, m2) == len(got)  # the size prepass
    tr.close()


def test_config1_queries(pst, oracle):
    """2^20 f32 points, dim1 ~ U[0,1000), dim2 = dim1 + U[0,50), ids 0..n-1: the
    3-sided (400, 420, 430) and 2-sided-left (500, 500) queries."""
    rng = np.random.default_rng(1)
    n = 1 << 20
    d1 = (rng.random(n, dtype=np.float32) * np.float32(1000)).astype(np.float32)
    d2 = (d1 + rng.random(n, dtype=np.float32) * np.float32(50)).astype(np.float32)
    pts = oracle.make_points(d1, d2, np.arange(n, dtype=np.uint32), "f32")
    ref = oracle.Orc.build(pts, "f32")
    tr = pst.StaticPSTGPU.from_numpy(pts, "f32")
    got3 = tr.threeSidedSearch(400, 420, 430, ret="ids")
    gotl = tr.twoSidedLeftSearch(500, 500, ret="ids")
    assert np.array_equal(oracle.canon(got3), oracle.canon(oracle.Orc.search_ids(ref, "three", 400, 420, 430)))
    assert np.array_equal(oracle.canon(gotl), oracle.canon(oracle.Orc.search_ids(ref, "left", 0, 500, 500)))
    brute3 = oracle.Orc.brute(pts, "f32", "three", 400, 420, 430)
    assert len(got3) == len(brute3) > 10000
    tr.close()


def test_extreme_bounds(pst, oracle):
    pts = rand_points(30000, "f32", ids="random", dup=True, seed=11)
    ref = oracle.Orc.build(pts, "f32")
    tr = pst.StaticPSTGPU.from_numpy(pts, "f32")
    inf = np.float32(np.inf)
    cases = [("three", -inf, inf, -inf), ("left", 0, inf, -inf), ("right", -inf, 0, -inf),
             ("three", 5, 1, -inf), ("left", 0, -inf, 0), ("right", inf, 0, 0), ("three", 0, 0, 0)]
    for kind, a, b, m2 in cases:
        got = tr.search(kind, a, b, m2, ret="ids")
        assert np.array_equal(oracle.canon(got), _oracle_set(oracle, ref, kind, a, b, m2, False)), (kind, a, b, m2)
    assert len(tr.search("three", -inf, inf, -inf)) == len(pts)
    tr.close()


def test_int_extremes(pst, oracle):
    rng = np.random.default_rng(5)
    n = 20000
    d1 = rng.integers(-2**31, 2**31 - 1, n, dtype=np.int64).astype(np.int32)
    d2 = np.maximum(d1, rng.integers(-2**31, 2**31 - 1, n, dtype=np.int64).astype(np.int32))
    d1[:5] = np.iinfo(np.int32).min
    d2[5:10] = np.iinfo(np.int32).max
    pts = oracle.make_points(d1, d2, rng.integers(0, 1000, n).astype(np.uint32), "i32")
    ref = oracle.Orc.build(pts, "i32")
    tr = pst.StaticPSTGPU.from_numpy(pts, "i32")
    assert tr.export()["dim1"].tobytes() == ref.dim1.tobytes()
    lo, hi = np.iinfo(np.int32).min, np.iinfo(np.int32).max
    for kind, a, b, m2 in [("three", lo, hi, lo), ("left", 0, 0, 0), ("right", 0, 0, hi), ("three", -5, 5, lo)]:
        got = tr.search(kind, a, b, m2)
        assert np.array_equal(oracle.canon(got), _oracle_set(oracle, ref, kind, a, b, m2, False))
    tr.close()


def test_search_into_capacity(pst, oracle):
    import torch
    pts = rand_points(10000, "f32", seed=3)
    tr = pst.StaticPSTGPU.from_numpy(pts, "f32")
    full = tr.search("left", 0, 600, 0)
    small = torch.empty(max(len(full) - 1, 1), dtype=torch.int32, device="cuda")
    assert tr.search_into("left", small, small.numel(), 0, 600, 0) == -len(full)
    big = torch.empty(len(full) + 5, dtype=torch.int32, device="cuda")
    assert tr.search_into("left", big, big.numel(), 0, 600, 0) == len(full)
    assert np.array_equal(np.sort(big[: len(full)].cpu().numpy().view(np.uint32)), np.sort(full))
    tr.close()


@pytest.mark.parametrize("dt", ["f32", "f64", "i32"])
@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_equals_single(pst, oracle, dt, use_graph):
    pts = rand_points(100000, dt, ids="random", dup=(dt == "i32"), seed=21)
    ref = oracle.Orc.build(pts, dt)
    tr = pst.StaticPSTGPU.from_numpy(pts, dt)
    qs = rand_queries(pts, 300, seed=22)
    q = pst.make_queries([pst.pst.KIND[k] for k, *_ in qs], [x[1] for x in qs], [x[2] for x in qs],
                         [x[3] for x in qs], dt)
    eng = pst.BatchEngine(tr, max_queries=512, task_capacity=1024, use_graph=use_graph)
    offs, res = eng.search(q)
    for i, (kind, a, b, m2) in enumerate(qs):
        got = res[offs[i]:offs[i + 1]]
        assert np.array_equal(oracle.canon(got), _oracle_set(oracle, ref, kind, a, b, m2, False)), i
    offs2, res2 = eng.search(q, ret="points")
    for i in range(0, len(qs), 7):
        kind, a, b, m2 = qs[i]
        got = res2[offs2[i]:offs2[i + 1]]
        assert np.array_equal(oracle.canon(got), _oracle_set(oracle, ref, kind, a, b, m2, True)), i
    eng.close()
    tr.close()


def test_batch_bad_kind_and_capacity(pst):
    import torch
    pts = rand_points(5000, "f32", seed=8)
    tr = pst.StaticPSTGPU.from_numpy(pts, "f32")
    eng = pst.BatchEngine(tr, max_queries=8)
    q = pst.make_queries([0, 1, 2], [0, 0, 0], [900, 900, 900], [0, 0, 0], "f32")
    counts, total = eng.count(q)
    assert total == int(counts.sum().item()) > 0
    out = torch.empty(16, dtype=torch.uint8, device="cuda")
    offs = torch.empty(4, dtype=torch.int64, device="cuda")
    st, tot = eng.run(q, out, offs)
    assert st == 4 and tot == total
    bad = q.copy()
    bad["kind"][1] = 9
    with pytest.raises(pst.PSTError):
        eng.count(bad)
    eng.close()
    tr.close()


def _narrow_queries(pts, k, seed):
    """k queries of a few results each: a 3-sided range around one point's dim1 with
    that point's dim2 as bound, and 2-sided ranges cut at the 6th smallest / largest
    dim1.  Their searches reach the bottom of the tree with a small frontier."""
    rng = np.random.default_rng(seed)
    d1, d2 = pts["dim1"], pts["dim2"]
    s1 = np.sort(d1)
    c = min(5, len(s1) - 1)
    out = []
    for j in range(k):
        i = int(rng.integers(0, len(pts)))
        kind = ["three", "left", "right"][j % 3]
        if kind == "three":
            out.append(("three", d1[i], d1[i], d2[i]))
        elif kind == "left":
            out.append(("left", 0, s1[c], rng.choice(d2)))
        else:
            out.append(("right", s1[-1 - c], 0, rng.choice(d2)))
    return out


@pytest.mark.parametrize("dt", ["f32", "f64", "i32"])
@pytest.mark.parametrize("use_graph", [True, False])
def test_small_batches(pst, oracle, dt, use_graph):
    """Batches of 1 to 33 queries (the top pass, which takes the upper levels in one
    CTA, serves batches of at most 32) into engines of 1 to 1024 queries: narrow
    queries whose frontier stays small to the bottom, wide ones that leave the lower
    levels to the per-level kernels, a mix of both, and a frontier buffer so small
    that the top pass overflows it and the engine grows it."""
    pts = rand_points(200003, dt, ids="random", dup=(dt == "i32"), seed=31)
    ref = oracle.Orc.build(pts, dt)
    tr = pst.StaticPSTGPU.from_numpy(pts, dt)
    narrow = _narrow_queries(pts, 33, seed=32)
    wide = rand_queries(pts, 33, seed=33)
    mixed = [narrow[i] if i % 2 else wide[i] for i in range(33)]
    want = {}
    for qs in (narrow, wide, mixed):
        for x in qs:
            if x not in want:
                want[x] = _oracle_set(oracle, ref, *x, False)
    for max_q, cap in ((1, 0), (32, 0), (33, 0), (1024, 0), (64, 64)):
        eng = pst.BatchEngine(tr, max_queries=max_q, task_capacity=cap, use_graph=use_graph)
        for qs in (narrow, wide, mixed):
            for nq in sorted({1, 2, 7, 31, 32, 33}):
                if nq > max_q:
                    continue
                sub = qs[:nq]
                q = pst.make_queries([pst.pst.KIND[k] for k, *_ in sub], [x[1] for x in sub], [x[2] for x in sub],
                                     [x[3] for x in sub], dt)
                counts, total = eng.count(q)
                offs, res = eng.search(q)
                assert offs[0] == 0 and int(offs[nq]) == total == len(res) == int(counts.sum().item())
                for i, x in enumerate(sub):
                    got = res[offs[i]:offs[i + 1]]
                    assert int(counts[i].item()) == len(got)
                    assert np.array_equal(oracle.canon(got), want[x]), (max_q, nq, i, x)
        eng.close()
    tr.close()


@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_async_run(pst, oracle, use_graph):
    """pst_batch_run with sync = 0 (everything enqueued, nothing waited for; small
    batches take the whole pass there) gives the offsets and results of the
    waiting run, for a small and a large batch."""
    import torch
    pts = rand_points(100000, "f32", ids="random", seed=41)
    ref = oracle.Orc.build(pts, "f32")
    tr = pst.StaticPSTGPU.from_numpy(pts, "f32")
    eng = pst.BatchEngine(tr, max_queries=512, use_graph=use_graph)
    for nq in (5, 300):
        qs = rand_queries(pts, nq, seed=42 + nq)
        q = pst.make_queries([pst.pst.KIND[k] for k, *_ in qs], [x[1] for x in qs], [x[2] for x in qs],
                             [x[3] for x in qs], "f32")
        offs, res = eng.search(q)
        out = torch.empty(max(len(res) * 4, 16), dtype=torch.uint8, device="cuda")
        offs_d = torch.empty(nq + 1, dtype=torch.int64, device="cuda")
        st, tot = eng.run(q, out, offs_d, sync=False)
        torch.cuda.synchronize()
        assert st == 0 and tot == len(res)
        assert np.array_equal(offs_d.cpu().numpy().astype(np.uint64), offs)
        got_all = out[: tot * 4].cpu().numpy().view(np.uint32)
        for i, x in enumerate(qs):
            got = got_all[offs[i]:offs[i + 1]]
            assert np.array_equal(oracle.canon(got), _oracle_set(oracle, ref, *x, False)), (nq, i)
    eng.close()
    tr.close()


@pytest.mark.parametrize("dt", ["f32", "i32"])
@pytest.mark.parametrize("n", [3, 63, 64, 65, 255, 256, 257, 511, 512, 513, 4095, 4096, 4097, 65535, 65536, 65537])
def test_batch_tree_sizes(pst, oracle, dt, n):
    """Batched search on trees whose last level is full, holds one node, or is
    missing (n = 2^k - 1, 2^k, 2^k + 1; the last-level parent bitmap exists from
    n = 256 on): a batch of 32 (top pass) and one of 60 (whole pass)."""
    pts = rand_points(n, dt, ids="random", dup=(dt == "i32"), seed=n + 77)
    ref = oracle.Orc.build(pts, dt)
    tr = pst.StaticPSTGPU.from_numpy(pts, dt)
    qs = rand_queries(pts, 30, seed=n) + _narrow_queries(pts, 30, seed=n + 1)
    eng = pst.BatchEngine(tr, max_queries=64)
    for sub in (qs[:32], qs):
        q = pst.make_queries([pst.pst.KIND[k] for k, *_ in sub], [x[1] for x in sub], [x[2] for x in sub],
                             [x[3] for x in sub], dt)
        offs, res = eng.search(q)
        for i, x in enumerate(sub):
            got = res[offs[i]:offs[i + 1]]
            assert np.array_equal(oracle.canon(got), _oracle_set(oracle, ref, *x, False)), (n, i, x)
    eng.close()
    tr.close()
