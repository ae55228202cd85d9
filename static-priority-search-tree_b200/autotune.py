"""Autotuner of the batched search: picks the launch shape of the level kernels
(CTAs per SM) and graph replay by timing candidates on a sample of the caller's own
queries, and caches the winner per (value type, tree levels, batch size,
selectivity decade) in a JSON file ($PST_AUTOTUNE_CACHE, default
~/.cache/pst_b200/autotune.json)."""
from __future__ import annotations

import json
import math
import os
import time
from pathlib import Path

import numpy as np

from .pst import BatchEngine, StaticPSTGPU

DEFAULT_CACHE = Path(os.environ.get("PST_AUTOTUNE_CACHE", Path.home() / ".cache" / "pst_b200" / "autotune.json"))


def cache_key(tree: StaticPSTGPU, nq: int, mean_count: float) -> str:
    levels = tree.info()["levels"]
    sel = mean_count / max(tree.n, 1)
    dec = int(math.floor(math.log10(sel))) if sel > 0 else -99
    return f"{tree.dt}-{'id' if tree.has_id else 'noid'}-L{levels}-q{int(math.log2(max(nq, 1)))}-s{dec}"


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


def tune(tree: StaticPSTGPU, queries: np.ndarray, candidates=(1, 2, 3, 4, 6, 8), repeats: int = 3,
         cache_path: Path | None = DEFAULT_CACHE, force: bool = False) -> dict:
    """Returns {"blocks_per_sm": b, "use_graph": g, "ms": t, "key": k}; the chosen
    configuration is the fastest mean of `repeats` timed passes over `queries`."""
    import torch
    nq = len(queries)
    probe = BatchEngine(tree, max_queries=nq)
    counts, total = probe.count(queries)
    probe.close()
    key = cache_key(tree, nq, total / max(nq, 1))
    cache = _load(cache_path) if cache_path else {}
    if not force and key in cache:
        return dict(cache[key], key=key, cached=True)
    out = torch.empty(max(total * (4 if tree.has_id else tree.rec_point.itemsize), 16), dtype=torch.uint8,
                      device="cuda")
    offs = torch.empty(nq + 1, dtype=torch.int64, device="cuda")
    qd = torch.from_numpy(np.ascontiguousarray(queries).view(np.uint8).copy()).to("cuda")
    ret = "ids" if tree.has_id else "points"
    best = None
    for use_graph in (True, False):
        for b in candidates:
            eng = BatchEngine(tree, max_queries=nq, blocks_per_sm=b, use_graph=use_graph)
            eng.run(qd, out, offs, ret=ret, queries_on_device=True, sync=True)  # sizes the frontier
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(repeats):
                eng.run(qd, out, offs, ret=ret, queries_on_device=True, sync=False)
            torch.cuda.synchronize()
            ms = (time.perf_counter() - t0) * 1000 / repeats
            eng.close()
            if best is None or ms < best["ms"]:
                best = {"blocks_per_sm": b, "use_graph": use_graph, "ms": ms}
    if cache_path:
        cache[key] = best
        _store(cache_path, cache)
    return dict(best, key=key, cached=False)
