"""Autotuner of the batched search.

The reference fixes one launch shape per query: a block of warp_multiplier x 32
threads walks the tree with a stack in shared memory
(pst/static-pst-gpu.tu:525-529).  Here a whole batch moves level by level, and the
launch shape is a set of choices the engine takes at creation (pst_batch_opts):

  * block_threads: CTA size of the level and emit kernels (128, 256, 512);
  * blocks_per_sm: level-kernel CTAs per SM (all that fit, or half of them);
  * emit_records: 64-slot records each emit warp keeps in flight (4, 8, 16: more
    loads in flight against more registers and fewer resident warps);
  * top_pass_queries: the largest waiting batch that starts with the one-CTA top
    pass, which walks the upper levels with the frontier kept by one CTA instead of
    a kernel launch per level (batches of up to 1024 queries: off, or the batch).

tune() times every combination on the caller's own queries (CUDA events around
passes over device-resident queries, after warm-up) and caches the fastest per
tree shape and batch size in a JSON file ($PST_AUTOTUNE_CACHE, default
~/.cache/pst_b200/autotune.json).  BatchEngine(tuning="cache") and
Server.add_tree(tuning="cache") read that cache.
"""
from __future__ import annotations

import itertools
import json
import math
import os
from pathlib import Path

import numpy as np

from .pst import BatchEngine, StaticPSTGPU

DEFAULT_CACHE = Path(os.environ.get("PST_AUTOTUNE_CACHE", Path.home() / ".cache" / "pst_b200" / "autotune.json"))
MAX_TOP_PASS = 1024


def cache_key(tree: StaticPSTGPU, nq: int) -> str:
    levels = tree.info()["levels"]
    return f"{tree.dt}-{'id' if tree.has_id else 'noid'}-L{levels}-q{int(math.log2(max(nq, 1)))}"


def _load(path: Path) -> dict:
    try:
        return json.loads(path.read_text())
    except Exception:
        return {}


def _store(path: Path, data: dict):
    try:
        path.parent.mkdir(parents=True, exist_ok=True)
        tmp = path.with_suffix(".tmp")
        tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
        tmp.replace(path)
    except OSError:
        pass


def cached(tree: StaticPSTGPU, nq: int, cache_path: Path | None = None) -> dict | None:
    """The cached choice for this tree shape and batch size, or None."""
    path = cache_path or DEFAULT_CACHE
    return _load(path).get(cache_key(tree, nq))


def candidates(nq: int, block_threads=(128, 256, 512), blocks_per_sm=(0, -2), emit_records=(4, 8, 16)):
    """The launch shapes tried for a batch of nq queries (blocks_per_sm -2 = half of
    what fits; it is resolved against the device when the engine is made)."""
    tops = (1, nq) if 1 < nq <= MAX_TOP_PASS else (0,)
    for bt, bps, er, tq in itertools.product(block_threads, blocks_per_sm, emit_records, tops):
        yield {"block_threads": bt, "blocks_per_sm": bps, "emit_records": er, "top_pass_queries": tq}


def _time(eng, qd, out, offs, ret, repeats, torch):
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    s = torch.cuda.current_stream()
    eng.run(qd, out, offs, ret=ret, queries_on_device=True, sync=True)  # sizes the frontier
    for _ in range(2):
        eng.run(qd, out, offs, ret=ret, queries_on_device=True, sync=False)
    torch.cuda.synchronize()
    ev[0].record(s)
    for _ in range(repeats):
        eng.run(qd, out, offs, ret=ret, queries_on_device=True, sync=False)
    ev[1].record(s)
    ev[1].synchronize()
    return ev[0].elapsed_time(ev[1]) / repeats


def tune(tree: StaticPSTGPU, queries: np.ndarray, repeats: int = 5, cache_path: Path | None = DEFAULT_CACHE,
         force: bool = False, task_capacity: int = 0, shapes=None) -> dict:
    """Times each launch shape on `queries` (a pst_query array) and returns the
    fastest: {block_threads, blocks_per_sm, emit_records, top_pass_queries,
    use_graph, ms, key, cached, tried: [(shape, ms), ...]}."""
    import torch
    nq = len(queries)
    key = cache_key(tree, nq)
    cache = _load(cache_path) if cache_path else {}
    if not force and key in cache:
        return dict(cache[key], key=key, cached=True)
    probe = BatchEngine(tree, max_queries=nq, task_capacity=task_capacity)
    _, total = probe.count(queries)
    probe.close()
    ret = "ids" if tree.has_id else "points"
    rec = 4 if tree.has_id else tree.rec_point.itemsize
    out = torch.empty(max(total * rec, 16), dtype=torch.uint8, device="cuda")
    offs = torch.empty(nq + 1, dtype=torch.int64, device="cuda")
    qd = torch.from_numpy(np.ascontiguousarray(queries).view(np.uint8).copy()).to("cuda")
    tried, best = [], None
    for shape in (shapes or candidates(nq)):
        shape = dict(shape)
        if shape["blocks_per_sm"] < 0:
            # half of what fits: an engine with the default reports the occupancy
            e0 = BatchEngine(tree, max_queries=nq, block_threads=shape["block_threads"], task_capacity=task_capacity)
            occ = e0.launch_shape()["blocks_per_sm"]
            e0.close()
            shape["blocks_per_sm"] = max(1, occ // 2)
        eng = BatchEngine(tree, max_queries=nq, task_capacity=task_capacity, tuning=shape)
        ms = _time(eng, qd, out, offs, ret, repeats, torch)
        eng.close()
        tried.append((shape, ms))
        if best is None or ms < best[1]:
            best = (shape, ms)
    result = dict(best[0], use_graph=True, ms=best[1])
    if cache_path:
        cache[key] = result
        _store(cache_path, cache)
    return dict(result, key=key, cached=False, tried=tried)

