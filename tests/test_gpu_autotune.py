"""Autotuner: times launch shapes on the caller's queries, returns a valid choice,
persists it, and serves the second call from the cache; the tuned engine's
results equal the default engine's."""
import numpy as np
import pytest

from datagen import rand_points, rand_queries

pytestmark = pytest.mark.gpu


def test_autotune_roundtrip(pst, tmp_path):
    import importlib
    at = importlib.import_module("pst_b200.autotune")
    pts = rand_points(200000, "f32", seed=41)
    tree = pst.StaticPSTGPU.from_numpy(pts, "f32")
    qs = rand_queries(pts, 64, seed=42)
    q = pst.make_queries([pst.pst.KIND[k] for k, *_ in qs], [x[1] for x in qs], [x[2] for x in qs],
                         [x[3] for x in qs], "f32")
    cache = tmp_path / "tune.json"
    best = at.tune(tree, q, candidates=(1, 4), repeats=2, cache_path=cache)
    assert best["blocks_per_sm"] in (1, 4) and best["ms"] > 0 and not best["cached"]
    again = at.tune(tree, q, candidates=(1, 4), cache_path=cache)
    assert again["cached"] and again["blocks_per_sm"] == best["blocks_per_sm"]
    eng = pst.BatchEngine(tree, max_queries=64, blocks_per_sm=best["blocks_per_sm"], use_graph=best["use_graph"])
    offs, res = eng.search(q)
    ref = pst.BatchEngine(tree, max_queries=64)
    offs2, res2 = ref.search(q)
    assert np.array_equal(offs, offs2)
    for i in range(len(qs)):
        assert np.array_equal(np.sort(res[offs[i]:offs[i + 1]]), np.sort(res2[offs2[i]:offs2[i + 1]]))
    eng.close()
    ref.close()
    tree.close()
