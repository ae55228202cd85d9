"""Autotuner and the launch shapes it chooses from: every shape (CTA size, level
CTAs per SM, emit records in flight, top-pass batch limit) returns the oracle's
results; tune() times the shapes on the caller's queries, returns one of them,
persists it and serves the next call from the cache; engines and servers built
from the cache use it; out-of-range shapes are rejected."""
import itertools

import numpy as np
import pytest

from datagen import rand_points, rand_queries

pytestmark = pytest.mark.gpu


def _queries(pst, pts, k, seed):
    qs = rand_queries(pts, k, seed=seed)
    q = pst.make_queries([pst.pst.KIND[x[0]] for x in qs], [x[1] for x in qs], [x[2] for x in qs],
                         [x[3] for x in qs], "f32")
    return qs, q


@pytest.mark.parametrize("ret", ["ids", "points"])
def test_every_launch_shape_matches_the_oracle(pst, oracle, ret):
    pts = rand_points(150001, "f32", ids="random", dup=True, seed=43)
    ref = oracle.Orc.build(pts, "f32")
    tree = pst.StaticPSTGPU.from_numpy(pts, "f32")
    qs, q = _queries(pst, pts, 300, 44)
    want = []
    for kind, a, b, m2 in qs:
        if ret == "ids":
            want.append(oracle.canon(oracle.Orc.search_ids(ref, kind, a, b, m2)))
        else:
            want.append(oracle.canon(oracle.Orc.search_points(ref, kind, a, b, m2)))
    for bt, er, tq, bps in itertools.product((128, 256, 512), (4, 8, 16), (0, 1024), (0, 1)):
        eng = pst.BatchEngine(tree, max_queries=len(qs), block_threads=bt, emit_records=er, top_pass_queries=tq,
                              blocks_per_sm=bps, task_capacity=4096)  # small frontier: growth on the way
        shape = eng.launch_shape()
        assert shape["block_threads"] == bt and shape["emit_records"] == er
        assert shape["top_pass_queries"] == (tq or 32)
        offs, res = eng.search(q, ret=ret)
        for i in range(len(qs)):
            got = res[int(offs[i]):int(offs[i + 1])]
            assert np.array_equal(oracle.canon(got), want[i]), (bt, er, tq, bps, i)
        eng.close()
    tree.close()


def test_rejects_out_of_range_shapes(pst):
    pts = rand_points(1000, "f32", seed=45)
    tree = pst.StaticPSTGPU.from_numpy(pts, "f32")
    for kw in ({"block_threads": 192}, {"emit_records": 5}, {"top_pass_queries": 4096}):
        with pytest.raises(pst.PSTError):
            pst.BatchEngine(tree, max_queries=4, **kw)
    tree.close()


def test_tune_caches_and_engines_use_the_cache(pst, tmp_path, monkeypatch):
    import importlib
    at = importlib.import_module("pst_b200.autotune")
    pts = rand_points(200000, "f32", seed=41)
    tree = pst.StaticPSTGPU.from_numpy(pts, "f32")
    qs, q = _queries(pst, pts, 64, 42)
    cache = tmp_path / "tune.json"
    shapes = [{"block_threads": 128, "blocks_per_sm": 0, "emit_records": 16, "top_pass_queries": 1},
              {"block_threads": 256, "blocks_per_sm": -2, "emit_records": 8, "top_pass_queries": 64}]
    best = at.tune(tree, q, repeats=2, cache_path=cache, shapes=shapes)
    assert not best["cached"] and best["ms"] > 0 and len(best["tried"]) == 2
    assert best["block_threads"] in (128, 256)
    again = at.tune(tree, q, cache_path=cache, shapes=shapes)
    assert again["cached"] and again["block_threads"] == best["block_threads"]
    monkeypatch.setattr(at, "DEFAULT_CACHE", cache)
    eng = pst.BatchEngine(tree, max_queries=64, tuning="cache")
    assert eng.launch_shape()["block_threads"] == best["block_threads"]
    assert eng.launch_shape()["emit_records"] == best["emit_records"]
    offs, res = eng.search(q)
    ref = pst.BatchEngine(tree, max_queries=64)
    offs2, res2 = ref.search(q)
    assert np.array_equal(offs, offs2)
    for i in range(len(qs)):
        assert np.array_equal(np.sort(res[offs[i]:offs[i + 1]]), np.sort(res2[offs2[i]:offs2[i + 1]]))
    # a server tree takes its engines' shape from the cache as well
    srv = pst.Server(max_batch=64, slots_per_tree=1, out_budget_bytes=1 << 26)
    idx = srv.add_tree(tree, tuning="cache")
    ids = srv.submit(idx, q[:8])
    for i, rid in enumerate(ids):
        got = srv.take(int(rid), np.uint32)
        assert np.array_equal(np.sort(got), np.sort(res2[offs2[i]:offs2[i + 1]]))
    srv.close()
    eng.close()
    ref.close()
    tree.close()
