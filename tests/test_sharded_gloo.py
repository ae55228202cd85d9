"""Multi-rank path on CPU: gloo ranks each hold one dim1 slab; routed queries and
the gathered results equal the single-tree answer.  Each rank's local search is
the oracle here (on GPUs it is the batch engine: tests/test_gpu_sharded.py); the
routing, the count all-gather and the point-to-point gather are the same code."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _load_sharded():
    import importlib.util
    spec = importlib.util.spec_from_file_location("sharded", ROOT / "static-priority-search-tree_b200" / "sharded.py")
    sh = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(sh)
    return sh


class OracleShard:
    """A shard whose local search is the CPU oracle (ids returned)."""

    def __init__(self, slab, dt, sh, oracle):
        self.oracle, self.dt = oracle, dt
        self.tree = oracle.Orc.build(slab, dt)
        self.bounds = sh.shard_ranges(slab)

    def record_size(self, ret):
        return 4

    def search(self, kinds, a, b, c, ret):
        import torch
        names = {0: "three", 1: "left", 2: "right"}
        outs = [self.oracle.Orc.search_ids(self.tree, names[int(k)], x, y, z) for k, x, y, z in zip(kinds, a, b, c)]
        offs = np.concatenate([[0], np.cumsum([len(o) for o in outs])]).astype(np.int64)
        recs = np.concatenate(outs).astype(np.uint32) if outs else np.zeros(0, np.uint32)
        return torch.from_numpy(offs), torch.from_numpy(recs.view(np.uint8).copy())


def _worker(rank, world, port, q, members):
    sys.path.insert(0, str(ROOT / "oracle"))
    sys.path.insert(0, str(ROOT / "tests"))
    import torch.distributed as dist
    from datagen import rand_points, rand_queries
    import oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sh = _load_sharded()
    # a subgroup (every rank creates it) or the default group
    group = dist.new_group(members) if members != list(range(world)) else None
    if rank in members:
        grank = members.index(rank)
        pts = rand_points(20000, "f32", ids="random", dup=True, seed=3)
        slab = sh.partition_by_dim1(pts, len(members))[grank]
        spst = sh.ShardedPST(OracleShard(slab, "f32", sh, oracle), group=group)
        qs = rand_queries(pts, 40, seed=4) + [("left", 0, 1e9, 1e9), ("three", 3, 2, -1e9)]
        kinds = np.array([sh.QUERY_KINDS[k] for k, *_ in qs])
        col = lambda j: np.array([x[j] for x in qs], np.float64)  # noqa: E731
        res = spst.search(kinds, col(1), col(2), col(3), dst=0)
        if grank == 0:
            ok = True
            offs, recs = res
            ids = recs.numpy().view(np.uint32)
            full = oracle.Orc.build(pts, "f32")
            for i, (kind, a, b, m2) in enumerate(qs):
                want = np.sort(oracle.Orc.search_ids(full, kind, np.float32(a), np.float32(b), np.float32(m2)))
                ok &= np.array_equal(np.sort(ids[int(offs[i]):int(offs[i + 1])]), want)
            # routing really prunes: a 3-sided query inside one slab visits one shard,
            # and a query above every shard's largest dim2 visits none
            lo0, hi0 = spst.ranges[0][:2]
            ok &= int(sh.route(0, lo0, (lo0 + hi0) / 2, spst.ranges).sum()) == 1
            ok &= int(sh.route(1, 0, 1e9, spst.ranges, min2=1e9).sum()) == 0
            q.put(bool(ok))
        else:
            assert res is None
    dist.barrier()
    dist.destroy_process_group()


def _run(world, members):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, members)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    assert all(p.exitcode == 0 for p in procs)
    assert q.get(timeout=5) is True


def test_two_rank_sharded_search():
    _run(2, [0, 1])


def test_sharded_search_on_a_subgroup():
    """Three ranks, the shards on group ranks 0 and 1 of the subgroup {1, 2}: sends
    and receives address peers by their global ranks."""
    _run(3, [1, 2])


def test_partition_and_route_host_logic():
    sys.path.insert(0, str(ROOT / "oracle"))
    sys.path.insert(0, str(ROOT / "tests"))
    from datagen import rand_points
    sh = _load_sharded()
    pts = rand_points(1001, "f32", ids="random", dup=True, seed=1)
    slabs = sh.partition_by_dim1(pts, 4)
    assert sum(len(s) for s in slabs) == 1001 and max(len(s) for s in slabs) - min(len(s) for s in slabs) <= 1
    for a, b in zip(slabs, slabs[1:]):
        assert a["dim1"].max() <= b["dim1"].min()
    ranges = np.array([sh.shard_ranges(s) for s in slabs])
    assert sh.route(1, 0, -1e9, ranges).sum() == 0
    assert sh.route(2, -1e9, 0, ranges).all()
    assert sh.route(0, 5, 4, ranges).sum() == 0
    # min2 above a shard's largest dim2 skips it
    top = ranges[:, 2]
    m = sh.route(1, 0, 1e9, ranges, min2=float(top[1]) + 1e-3)
    assert m.tolist() == [bool(t > top[1] + 1e-3) for t in top]
    # an empty shard is never visited
    ranges2 = np.vstack([ranges, [np.inf, -np.inf, -np.inf, 0.0]])
    assert not sh.route(2, -1e9, 0, ranges2)[-1]
    # route_many agrees with route query by query
    rng = np.random.default_rng(2)
    k = rng.integers(0, 3, 50)
    a, b, c = (rng.uniform(-20, 20, 50) for _ in range(3))
    many = sh.route_many(k, a, b, c, ranges)
    for i in range(50):
        assert np.array_equal(many[i], sh.route(int(k[i]), a[i], b[i], ranges, min2=c[i]))
