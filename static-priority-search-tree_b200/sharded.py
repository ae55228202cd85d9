"""Sharded priority search tree: one dim1 slab per rank (one process per GPU).

The points are cut into contiguous dim1 ranges (slabs of the reference's dim1
order: value, then id, then input index) and each rank builds the tree of its slab
with the GPU engine.  A query visits only the shards that can hold a result: a
shard's (min dim1, max dim1, max dim2) bound its points, so a 3-sided query needs
[min1, max1] to meet [lo, hi], a 2-sided-left query lo <= max1, a 2-sided-right
query hi >= min1, and every kind max dim2 >= min2.  Every point lives on one
shard, so a query's result is the concatenation of its shards' results, and a
search needs no exchange at all; gathering the results to one rank is optional:
the per-query counts of every rank in one all-gather, then each rank's records in
one point-to-point message (device tensors on an NCCL group, so the records cross
NVLink into the receiver's HBM; host tensors on gloo).  Nothing here reads another
GPU's memory directly: every transfer is an NCCL (or gloo) message.

The reference has no multi-GPU search (its dev_ind / num_devs arguments only appear
in messages, pst/static-pst-gpu.tu:62-63); this is the sharding of its searches
(pst/static-pst-gpu.tu:496-642) by dim1 ranges.
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
    """(min dim1, max dim1, max dim2, nonempty) of one host slab as float64."""
    if len(slab) == 0:
        return (np.inf, -np.inf, -np.inf, 0.0)
    return (float(slab["dim1"].min()), float(slab["dim1"].max()), float(slab["dim2"].max()), 1.0)


def route_many(kinds, min1, max1, min2, ranges: np.ndarray) -> np.ndarray:
    """(nq, shards) mask of the shards each query must visit; ranges[r] = (min dim1,
    max dim1, max dim2, nonempty).  Comparisons run in float64, which holds every
    float32, int32 and float64 bound exactly."""
    k = np.asarray(kinds)[:, None]
    a = np.asarray(min1, np.float64)[:, None]
    b = np.asarray(max1, np.float64)[:, None]
    c = np.asarray(min2, np.float64)[:, None]
    lo, hi, top, ne = (ranges[None, :, i] for i in range(4))
    three = (hi >= a) & (lo <= b) & (a <= b)  # min1 > max1 matches no point
    left = lo <= b
    right = hi >= a
    hit = np.where(k == 0, three, np.where(k == 1, left, right))
    return hit & (top >= c) & (ne > 0)


def route(kind: int, min1: float, max1: float, ranges: np.ndarray, min2: float = -np.inf) -> np.ndarray:
    """Mask of the shards one query must visit (route_many for a single query)."""
    return route_many([kind], [min1], [max1], [min2], ranges)[0]


class GpuShard:
    """The local slab's tree and batch engine (the GPU path of a shard)."""

    def __init__(self, pst, slab_d, n: int, dt: str = "f32", has_id: bool = True, max_queries: int = 4096):
        import torch
        self.pst, self.torch = pst, torch
        self.dt, self.has_id, self.n = dt, has_id, int(n)
        self.tree = pst.StaticPSTGPU(slab_d, self.n, dt, has_id)
        self.max_queries = max_queries
        self.eng = pst.BatchEngine(self.tree, max_queries=max_queries)
        self.rec_point = pst.point_dtype(dt, has_id)
        self.bounds = self._device_bounds(slab_d)

    def _device_bounds(self, slab_d):
        torch = self.torch
        if self.n == 0:
            return (np.inf, -np.inf, -np.inf, 0.0)
        vt = {"f32": torch.float32, "f64": torch.float64, "i32": torch.int32}[self.dt]
        vs = 8 if self.dt == "f64" else 4
        words = slab_d.reshape(-1).view(torch.uint8)[: self.n * self.rec_point.itemsize].view(vt)
        cols = words.reshape(self.n, self.rec_point.itemsize // vs)
        d1, d2 = cols[:, 0], cols[:, 1]
        return (float(d1.min().item()), float(d1.max().item()), float(d2.max().item()), 1.0)

    def record_size(self, ret: str) -> int:
        return 4 if ret == "ids" else self.rec_point.itemsize

    def search(self, kinds, min1, max1, min2, ret="ids"):
        """Routed queries on the local tree: (offsets[nq + 1] int64, records uint8)
        as device tensors, in batches of at most max_queries."""
        torch = self.torch
        nq = len(kinds)
        rsz = self.record_size(ret)
        offs_all, parts, base = [torch.zeros(1, dtype=torch.int64, device="cuda")], [], 0
        for s in range(0, nq, self.max_queries):
            e = min(nq, s + self.max_queries)
            q = self.pst.make_queries(kinds[s:e], min1[s:e], max1[s:e], min2[s:e], self.dt)
            _, total = self.eng.count(q)
            out = torch.empty(max(total * rsz, 16), dtype=torch.uint8, device="cuda")
            offs = torch.empty(e - s + 1, dtype=torch.int64, device="cuda")
            st, tot = self.eng.run(q, out, offs, ret=ret)
            if st != 0:
                raise RuntimeError(f"shard search failed with status {st}")
            offs_all.append(offs[1:] + base)
            parts.append(out[: tot * rsz])
            base += tot
        offsets = torch.cat(offs_all)
        records = torch.cat(parts) if parts else torch.zeros(0, dtype=torch.uint8, device="cuda")
        return offsets, records

    def close(self):
        self.eng.close()
        self.tree.close()


class ShardedPST:
    """One shard per rank of a torch.distributed process group.

    `local` answers the queries routed to this rank: an object with
    search(kinds, min1, max1, min2, ret) -> (offsets[nq + 1], records as bytes),
    record_size(ret), its value type `dt` and `bounds` = (min dim1, max dim1, max
    dim2, nonempty) of its slab (GpuShard on a GPU; the CPU tests pass an
    oracle-backed one)."""

    def __init__(self, local, group=None):
        import torch
        import torch.distributed as dist
        self.dist, self.torch, self.group = dist, torch, group
        self.local = local
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.dev = torch.device("cuda") if dist.get_backend(group) == "nccl" else torch.device("cpu")
        mine = torch.tensor(local.bounds, dtype=torch.float64, device=self.dev)
        allr = [torch.zeros(4, dtype=torch.float64, device=self.dev) for _ in range(self.world)]
        dist.all_gather(allr, mine, group=group)
        self.ranges = torch.stack(allr).cpu().numpy()

    def _peer(self, r: int) -> int:
        """Global rank of group rank r (send / recv address peers by global rank)."""
        if self.group is None or self.group == self.dist.group.WORLD:
            return r
        return self.dist.get_global_rank(self.group, r)

    def routed(self, kinds, min1, max1, min2) -> np.ndarray:
        """Indices of the queries this rank answers."""
        return np.nonzero(route_many(kinds, min1, max1, min2, self.ranges)[:, self.rank])[0]

    def search_local(self, kinds, min1, max1, min2, ret="ids"):
        """The shard's part of every query, with no exchange: (per-query counts [nq]
        int64, records) on this rank's device; the records of query i are this
        shard's results of query i, in query order."""
        torch = self.torch
        kinds = np.asarray(kinds)
        nq = len(kinds)
        # route on the bounds the shard searches with (the tree's value type)
        vt = {"f32": np.float32, "f64": np.float64, "i32": np.int32}[self.local.dt]
        min1, max1, min2 = (np.asarray(x).astype(vt) for x in (min1, max1, min2))
        sel = self.routed(kinds, min1, max1, min2)
        counts = torch.zeros(nq, dtype=torch.int64, device=self.dev)
        if len(sel) == 0:
            return counts, torch.zeros(0, dtype=torch.uint8, device=self.dev)
        offs, recs = self.local.search(kinds[sel], np.asarray(min1)[sel], np.asarray(max1)[sel],
                                       np.asarray(min2)[sel], ret)
        offs = torch.as_tensor(offs).to(self.dev)
        counts[torch.as_tensor(sel, device=self.dev)] = offs[1:] - offs[:-1]
        return counts, torch.as_tensor(recs).to(self.dev)

    def search(self, kinds, min1, max1, min2, ret="ids", dst: int = 0):
        """Runs the queries (the same list on every rank) and gathers the results on
        group rank `dst`, which receives (offsets[nq + 1] int64, records uint8) on its
        device, query i's records at [offsets[i], offsets[i + 1]) (shard order inside
        a query); the other ranks return None.  Every rank takes the same collective
        steps whatever its share of the work."""
        torch, dist = self.torch, self.dist
        nq = len(kinds)
        rsz = self.local.record_size(ret)
        counts, recs = self.search_local(kinds, min1, max1, min2, ret)
        all_ct = [torch.zeros(nq, dtype=torch.int64, device=self.dev) for _ in range(self.world)]
        dist.all_gather(all_ct, counts, group=self.group)
        C = torch.stack(all_ct)  # (shards, queries)
        totals = C.sum(dim=1).tolist()
        if self.rank != dst:
            if totals[self.rank]:
                req = dist.isend(recs[: totals[self.rank] * rsz].contiguous(), dst=self._peer(dst), group=self.group)
                req.wait()
            return None
        bufs, ops = [], []
        for r in range(self.world):
            if r == self.rank:
                bufs.append(recs[: totals[r] * rsz])
                continue
            b = torch.empty(totals[r] * rsz, dtype=torch.uint8, device=self.dev)
            bufs.append(b)
            if totals[r]:
                ops.append(dist.P2POp(dist.irecv, b, self._peer(r), self.group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        # query i's records: shard 0's, then shard 1's, ... at the global offsets
        per_q = C.sum(dim=0)
        offsets = torch.zeros(nq + 1, dtype=torch.int64, device=self.dev)
        offsets[1:] = torch.cumsum(per_q, 0)
        before = torch.cumsum(C, 0) - C  # records of query i on the shards before r
        out = torch.empty(int(offsets[-1].item()) * rsz, dtype=torch.uint8, device=self.dev)
        qidx = torch.arange(nq, device=self.dev)
        for r in range(self.world):
            if not totals[r]:
                continue
            q_of = torch.repeat_interleave(qidx, C[r])
            loff = torch.cumsum(C[r], 0) - C[r]
            j = torch.arange(totals[r], device=self.dev)
            dest = offsets[q_of] + before[r, q_of] + (j - loff[q_of])
            out.view(-1, rsz)[dest] = bufs[r].view(-1, rsz)
        return offsets, out
