"""Sharded priority search tree over ranks (one process per GPU).

Points are split into contiguous dim1 ranges (cut from the global dim1 order), each
rank builds the tree of its slab, and a query only visits the shards whose dim1
range it can touch: a 3-sided query the shards meeting [min1, max1], a 2-sided-left
query those with some dim1 <= max1, a 2-sided-right query those with some
dim1 >= min1.  Every point lives on one shard, so a query's result is the
concatenation of its shards' results; the only exchange is the gather of those
variable-length results to one rank (counts first, then the records).

The local search is a callable (the GPU batch engine in production), so the
routing and exchange logic is the same whatever runs it.
"""
from __future__ import annotations

import numpy as np

QUERY_KINDS = {"three": 0, "left": 1, "right": 2}


def partition_by_dim1(points: np.ndarray, world: int) -> list[np.ndarray]:
    """Splits PointStruct records into `world` slabs of (nearly) equal size by the
    reference's dim1 order (value, then id, then input index)."""
    keys = [points["dim1"]]
    order = np.lexsort(([np.arange(len(points))] + ([points["id"]] if "id" in points.dtype.names else [])
                        + keys)) if len(points) else np.zeros(0, np.int64)
    cuts = np.linspace(0, len(points), world + 1).astype(np.int64)
    return [points[order[cuts[r]:cuts[r + 1]]] for r in range(world)]


def shard_ranges(slab: np.ndarray):
    """(min dim1, max dim1, nonempty) of one slab as float64."""
    if len(slab) == 0:
        return (np.inf, -np.inf, 0.0)
    return (float(slab["dim1"].min()), float(slab["dim1"].max()), 1.0)


def route(kind: int, min1: float, max1: float, ranges: np.ndarray) -> np.ndarray:
    """Boolean mask of the shards a query must visit.  ranges[r] = (lo, hi, nonempty)."""
    lo, hi, ne = ranges[:, 0], ranges[:, 1], ranges[:, 2] > 0
    if kind == 0:
        # min1 > max1 matches no point (min1 <= dim1 <= max1 is unsatisfiable)
        hit = (hi >= min1) & (lo <= max1) & (min1 <= max1)
    elif kind == 1:
        hit = lo <= max1
    else:
        hit = hi >= min1
    return hit & ne


class ShardedPST:
    """One shard per rank of a torch.distributed process group.

    local_search(kinds, min1, max1, min2) -> (offsets[nq + 1], results) runs the
    queries routed to this rank on the local slab (uint32 ids)."""

    def __init__(self, slab: np.ndarray, local_search, group=None):
        import torch
        import torch.distributed as dist
        self.dist, self.torch, self.group = dist, torch, group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.local_search = local_search
        mine = torch.tensor(shard_ranges(slab), dtype=torch.float64)
        allr = [torch.zeros(3, dtype=torch.float64) for _ in range(self.world)]
        dist.all_gather(allr, mine, group=group)
        self.ranges = torch.stack(allr).numpy()

    def search(self, kinds, min1, max1, min2, dst: int = 0):
        """Runs the queries (the same list on every rank); rank `dst` receives a list
        of per-query id arrays, the other ranks None."""
        torch, dist = self.torch, self.dist
        kinds = np.asarray(kinds)
        nq = len(kinds)
        mask = np.array([route(int(kinds[i]), float(min1[i]), float(max1[i]), self.ranges)[self.rank]
                         for i in range(nq)], bool)
        sel = np.nonzero(mask)[0]
        counts = np.zeros(nq, np.int64)
        res = np.zeros(0, np.uint32)
        if len(sel):
            offs, res = self.local_search(kinds[sel], np.asarray(min1)[sel], np.asarray(max1)[sel],
                                          np.asarray(min2)[sel])
            counts[sel] = np.diff(np.asarray(offs, np.int64))
        # exchange: per-query counts of every rank, then the variable-length records
        ct = torch.from_numpy(counts)
        all_ct = [torch.zeros(nq, dtype=torch.int64) for _ in range(self.world)]
        dist.all_gather(all_ct, ct, group=self.group)
        totals = [int(c.sum()) for c in all_ct]
        if self.rank == dst:
            parts = []
            for r in range(self.world):
                if r == dst:
                    parts.append(res.astype(np.int64))
                    continue
                buf = torch.zeros(totals[r], dtype=torch.int64)
                if totals[r]:
                    dist.recv(buf, src=r, group=self.group)
                parts.append(buf.numpy())
            out = []
            starts = [np.concatenate([[0], np.cumsum(all_ct[r].numpy())]) for r in range(self.world)]
            for i in range(nq):
                pieces = [parts[r][starts[r][i]:starts[r][i + 1]] for r in range(self.world)]
                out.append(np.concatenate(pieces).astype(np.uint32) if pieces else np.zeros(0, np.uint32))
            return out
        if totals[self.rank]:
            dist.send(torch.from_numpy(res.astype(np.int64)), dst=dst, group=self.group)
        return None
