"""Parity at the benchmarked sizes: results of the large configurations, checked id
by id against the oracle's brute force (the query predicates of
pst/static-pst-cpu-iter.tpp:247-251, :355-358, :446-449, evaluated over every point
by orc_brute_multi, threaded C).

* the batched step of the benchmark itself: 2^28 float32 points with ids,
  dim1 ~ U[0, 2^24), dim2 = dim1 + U[0, 2^16), its 4096 calibrated queries (50 %
  3-sided, 25 % left, 25 % right, selectivities log-uniform in [1e-7, 1e-2]);
  64 of them, the 16 largest among them, compared with brute force, and every
  256th query's count compared with the plain per-query count;
* the batched-queries configuration: 2^26 float32 points, dim1 ~ U[0, 1),
  dim2 = dim1 + Exp(mean 0.01), 4096 queries of the same mix; a sample of 256
  compared with brute force (dim1 is drawn on a grid of 2^-24, so every value is
  shared by four points on average: ties everywhere);
* the large random trees in float64 and int32 (and float32 without ids,
  returning whole points) at 2^26 points: each kind at selectivities 1e-5, 1e-3
  and 1e-1, batched and plain.

Paths that only occur at these sizes are exercised here: 27-29 tree levels,
frontiers of millions of records, multi-GB outputs with 64-bit offsets.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
import bench  # noqa: E402

pytestmark = pytest.mark.gpu

KIND_NAMES = {0: "three", 1: "left", 2: "right"}


def _device_records_to_host(rec, dt, has_id, oracle):
    """A (n, k) device tensor of PointStruct words -> structured host array."""
    host = rec.cpu().numpy()
    return host.view(np.uint8).reshape(-1).view(oracle.point_dtype(dt, has_id))


def _batched_results(pst, torch, eng, q_host, ret, rec_bytes):
    counts, total = eng.count(q_host)
    q_dev = torch.from_numpy(q_host.view(np.uint8).copy()).to("cuda")
    out = torch.empty(total * rec_bytes + 16, dtype=torch.uint8, device="cuda")
    offs = torch.empty(len(q_host) + 1, dtype=torch.int64, device="cuda")
    st, tot = eng.run(q_dev, out, offs, ret=ret, queries_on_device=True, sync=True)
    assert st == 0 and tot == total
    return out, offs.cpu().numpy().astype(np.int64), counts.cpu().numpy()


def _check_sample(oracle, pts_host, dt, q_host, sample, out, offs, rec_bytes, ret):
    """Sorted GPU ids (or point records) of the sampled queries == brute force."""
    kinds = q_host["kind"][sample]
    vals = {}
    for f in ("min1", "max1", "min2"):
        raw = np.ascontiguousarray(q_host[f][sample]).view(np.uint8).reshape(-1, 8)
        vals[f] = np.ascontiguousarray(raw[:, : np.dtype(oracle.DTYPES[dt]).itemsize]).view(oracle.DTYPES[dt])[:, 0]
    boff, bidx = oracle.Orc.brute_multi(pts_host, dt, kinds, vals["min1"], vals["max1"], vals["min2"])
    for j, i in enumerate(sample):
        lo, hi = int(offs[i]), int(offs[i + 1])
        got = out[lo * rec_bytes: hi * rec_bytes].cpu().numpy()
        want_idx = bidx[int(boff[j]): int(boff[j + 1])]
        assert hi - lo == len(want_idx), (int(i), KIND_NAMES[int(kinds[j])], hi - lo, len(want_idx))
        if ret == "ids":
            want = np.sort(pts_host["id"][want_idx].astype(np.uint64))
            assert np.array_equal(np.sort(got.view(np.uint32).astype(np.uint64)), want), int(i)
        else:
            want = oracle.canon(pts_host[want_idx])
            assert np.array_equal(oracle.canon(got.view(pts_host.dtype)), want), int(i)


def _sample(counts, k_largest, k_total, seed):
    order = np.argsort(counts)[::-1]
    big = order[:k_largest]
    rest = np.setdiff1d(np.arange(len(counts)), big)
    pick = np.random.default_rng(seed).choice(rest, k_total - k_largest, replace=False)
    return np.sort(np.concatenate([big, pick]))


def test_benchmark_step_2p28(pst, oracle):
    """The benchmark's own workload (bench.py's generators, plan and calibration)."""
    import torch
    n = bench.N_POINTS
    rec = bench.gen_points_device(n, seed=1, torch=torch)
    tree = pst.StaticPSTGPU(rec, n, "f32", True)
    assert tree.info()["levels"] == 29
    eng = pst.BatchEngine(tree, max_queries=bench.NQ, task_capacity=n >> 2)
    kinds, sel, anchor = bench.query_plan(bench.NQ, 7)

    def count_fn(k, a, b, c):
        return eng.count(pst.make_queries(k, a, b, c, "f32"))[0].cpu().numpy()
    min1, max1, min2 = bench.calibrate(count_fn, kinds, sel, anchor, n)
    q_host = pst.make_queries(kinds, min1, max1, min2, "f32")
    out, offs, counts = _batched_results(pst, torch, eng, q_host, "ids", 4)
    assert offs[-1] > 500_000_000  # the step reports close to a billion points
    pts_host = _device_records_to_host(rec, "f32", True, oracle)
    del rec
    sample = _sample(counts, 16, 64, seed=5)
    _check_sample(oracle, pts_host, "f32", q_host, sample, out, offs, 4, "ids")
    # every query's size from the plain per-query prepass equals the batched count
    for i in range(0, bench.NQ, 256):
        assert tree.count(KIND_NAMES[int(kinds[i])], min1[i], max1[i], min2[i]) == int(counts[i]), i
    del out
    eng.close()
    tree.close()
    torch.cuda.empty_cache()


def test_batched_queries_config_2p26_exp(pst, oracle):
    """2^26 points, dim1 ~ U[0,1), dim2 = dim1 + Exp(mean 0.01); 4096 mixed queries."""
    import torch
    n = 1 << 26
    rec = bench.gen_points_exp_device(n, seed=3, torch=torch)
    tree = pst.StaticPSTGPU(rec, n, "f32", True)
    eng = pst.BatchEngine(tree, max_queries=bench.NQ, task_capacity=n >> 2)
    kinds, sel, anchor = bench.query_plan(bench.NQ, 9)
    anchor = anchor / float(1 << 24)

    def count_fn(k, a, b, c):
        return eng.count(pst.make_queries(k, a, b, c, "f32"))[0].cpu().numpy()
    min1, max1, min2 = bench.calibrate(count_fn, kinds, sel, anchor, n, domain=1.0, spread=0.25)
    q_host = pst.make_queries(kinds, min1, max1, min2, "f32")
    out, offs, counts = _batched_results(pst, torch, eng, q_host, "ids", 4)
    # calibration reached its targets (log-uniform sizes from a handful of points up)
    big = sel * n > 1000
    assert np.median(np.abs(counts[big] - sel[big] * n) / (sel[big] * n)) < 0.02
    pts_host = _device_records_to_host(rec, "f32", True, oracle)
    del rec
    sample = _sample(counts, 16, 256, seed=6)
    _check_sample(oracle, pts_host, "f32", q_host, sample, out, offs, 4, "ids")
    del out
    eng.close()
    tree.close()
    torch.cuda.empty_cache()


def _typed_queries(dt, n, seed):
    """Each kind at selectivities 1e-5, 1e-3 and 1e-1 (approximate: bounds set from
    the distribution, dim1 ~ U[0, 2^24), dim2 = dim1 + U[0, 2^16)), two anchors each."""
    rng = np.random.default_rng(seed)
    D, w = float(1 << 24), float(1 << 16)
    rows = []
    for kind in (0, 1, 2):
        for s in (1e-5, 1e-3, 1e-1):
            for _ in range(2):
                W = s * D
                if kind == 0:
                    a = rng.uniform(0, D - W)
                    rows.append((0, a, a + W, a))
                elif kind == 1:
                    b = rng.uniform(W + w, D)
                    rows.append((1, 0.0, b, b - W + w / 2))
                else:
                    a = D - W - w / 2 - rng.uniform(0, W / 4)
                    rows.append((2, a, 0.0, a))
    k = np.array([r[0] for r in rows], np.int32)
    cols = [np.array([r[i] for r in rows]) for i in (1, 2, 3)]
    if dt == "i32":
        cols = [np.round(c).astype(np.int32) for c in cols]
    return k, cols


@pytest.mark.parametrize("dt,has_id", [("f64", True), ("i32", True), ("f32", False)])
def test_large_random_trees_2p26(pst, oracle, dt, has_id):
    import torch
    n = 1 << 26
    rec = bench.gen_points_typed(n, 1, dt, has_id, torch)
    tree = pst.StaticPSTGPU(rec, n, dt, has_id)
    kinds, (min1, max1, min2) = _typed_queries(dt, n, seed=8)
    q_host = pst.make_queries(kinds, min1, max1, min2, dt)
    ret = "ids" if has_id else "points"
    pts_dtype = oracle.point_dtype(dt, has_id)
    rec_bytes = 4 if has_id else pts_dtype.itemsize
    eng = pst.BatchEngine(tree, max_queries=len(kinds), task_capacity=n >> 2)
    out, offs, counts = _batched_results(pst, torch, eng, q_host, ret, rec_bytes)
    assert counts.max() > n // 20  # the 1e-1 queries really are large
    pts_host = _device_records_to_host(rec, dt, has_id, oracle)
    del rec
    _check_sample(oracle, pts_host, dt, q_host, np.arange(len(kinds)), out, offs, rec_bytes, ret)
    # the plain drop-in path on the small and middle selectivities
    for i in range(len(kinds)):
        if counts[i] > n // 100:
            continue
        got = tree.search(KIND_NAMES[int(kinds[i])], min1[i], max1[i], min2[i], ret=ret)
        lo, hi = int(offs[i]), int(offs[i + 1])
        batched = out[lo * rec_bytes: hi * rec_bytes].cpu().numpy()
        if has_id:
            assert np.array_equal(np.sort(got), np.sort(batched.view(np.uint32)))
        else:
            assert np.array_equal(oracle.canon(got), oracle.canon(batched.view(pts_dtype)))
    del out
    eng.close()
    tree.close()
    torch.cuda.empty_cache()


def test_top_pass_large_limit_2p25(pst, oracle):
    """Small batches on a deep tree with the largest top-pass batch limit (1024, so
    the one-CTA pass keeps 4 x 2048 path and seed slots and ~5300 records in shared
    memory): batches of 40 … 240 tiny queries run the top pass over most of the 26
    levels and hand their records, paths and seeds over to the level kernels where
    a level first holds more than 256 records.  Every query is checked against brute
    force.  (The record array's own bound, checked before each level, is a safety
    net: records grow about geometrically with depth, so a level exceeds 256 records
    before the levels above it fill the array.)"""
    import torch
    n = 1 << 25
    rec = bench.gen_points_device(n, seed=4, torch=torch)
    tree = pst.StaticPSTGPU(rec, n, "f32", True)
    assert tree.info()["levels"] == 26
    pts_host = _device_records_to_host(rec, "f32", True, oracle)
    del rec
    eng = pst.BatchEngine(tree, max_queries=1024, task_capacity=1 << 22, top_pass_queries=1024)
    rng = np.random.default_rng(11)
    D, w = float(1 << 24), float(1 << 16)
    for nq in (40, 80, 120, 160, 240):
        kinds = np.where(np.arange(nq) % 2 == 0, 0, 1).astype(np.int32)
        a = rng.uniform(w, D - w, nq)
        width = rng.uniform(4.0, 40.0, nq)
        min1 = np.where(kinds == 0, a, 0.0)
        max1 = np.where(kinds == 0, a + width, a)
        min2 = np.where(kinds == 0, a, a + w - width)  # left: only points within ~width of max1 reach min2
        q_host = pst.make_queries(kinds, min1.astype(np.float32), max1.astype(np.float32),
                                  min2.astype(np.float32), "f32")
        out, offs, counts = _batched_results(pst, torch, eng, q_host, "ids", 4)
        assert counts.sum() > 0
        _check_sample(oracle, pts_host, "f32", q_host, np.arange(nq), out, offs, 4, "ids")
        del out
    eng.close()
    tree.close()
    torch.cuda.empty_cache()
