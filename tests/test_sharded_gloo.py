"""Multi-rank path on CPU: two gloo ranks each hold one dim1 slab; routed queries
and the gathered results equal the single-tree answer (the oracle runs each
rank's local search here; on GPUs it is the batch engine)."""
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


def _worker(rank, world, port, q):
    sys.path.insert(0, str(ROOT / "oracle"))
    sys.path.insert(0, str(ROOT / "tests"))
    import importlib.util

    import torch.distributed as dist
    from datagen import rand_points, rand_queries
    import oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    spec = importlib.util.spec_from_file_location("sharded", ROOT / "static-priority-search-tree_b200" / "sharded.py")
    sh = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(sh)
    pts = rand_points(20000, "f32", ids="random", dup=True, seed=3)
    slab = sh.partition_by_dim1(pts, world)[rank]
    tree = oracle.Orc.build(slab, "f32")
    names = {0: "three", 1: "left", 2: "right"}

    def local(kinds, a, b, c):
        outs = [oracle.Orc.search_ids(tree, names[int(k)], x, y, z) for k, x, y, z in zip(kinds, a, b, c)]
        offs = np.concatenate([[0], np.cumsum([len(o) for o in outs])])
        return offs, (np.concatenate(outs) if outs else np.zeros(0, np.uint32))

    spst = sh.ShardedPST(slab, local)
    qs = rand_queries(pts, 40, seed=4)
    kinds = np.array([sh.QUERY_KINDS[k] for k, *_ in qs])
    res = spst.search(kinds, [x[1] for x in qs], [x[2] for x in qs], [x[3] for x in qs])
    ok = True
    if rank == 0:
        full = oracle.Orc.build(pts, "f32")
        for i, (kind, a, b, m2) in enumerate(qs):
            want = np.sort(oracle.Orc.search_ids(full, kind, a, b, m2))
            ok &= np.array_equal(np.sort(res[i]), want)
        # routing really prunes: a 3-sided query inside one slab visits one shard
        lo0, hi0 = spst.ranges[0][:2]
        mid = (lo0 + hi0) / 2
        ok &= int(sh.route(0, lo0, mid, spst.ranges).sum()) == 1
        q.put(bool(ok))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharded_search():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    assert all(p.exitcode == 0 for p in procs)
    assert q.get(timeout=5) is True


def test_partition_and_route_host_logic():
    import importlib.util
    sys.path.insert(0, str(ROOT / "oracle"))
    sys.path.insert(0, str(ROOT / "tests"))
    from datagen import rand_points
    spec = importlib.util.spec_from_file_location("sharded", ROOT / "static-priority-search-tree_b200" / "sharded.py")
    sh = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(sh)
    pts = rand_points(1001, "f32", ids="random", dup=True, seed=1)
    slabs = sh.partition_by_dim1(pts, 4)
    assert sum(len(s) for s in slabs) == 1001 and max(len(s) for s in slabs) - min(len(s) for s in slabs) <= 1
    for a, b in zip(slabs, slabs[1:]):
        assert a["dim1"].max() <= b["dim1"].min()
    ranges = np.array([sh.shard_ranges(s) for s in slabs])
    assert sh.route(1, 0, -1e9, ranges).sum() == 0
    assert sh.route(2, -1e9, 0, ranges).all()
    assert sh.route(0, 5, 4, ranges).sum() == 0
