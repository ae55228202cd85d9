"""The sharded search with the GPU engine on every shard: two ranks (gloo, both on
cuda:0, which is all a single-GPU run has), each holding one dim1 slab as a GPU
tree; queries routed by the slabs' bounds, each shard's part run by its batch
engine, the results gathered to rank 0, and every query's gathered ids equal to
the oracle's answer on the whole point set.  The ranks' kernels never wait on one
another: the only exchange is host-side (gloo)."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q, dt):
    sys.path.insert(0, str(ROOT / "oracle"))
    sys.path.insert(0, str(ROOT / "tests"))
    import torch
    import torch.distributed as dist
    from conftest import load_package
    from datagen import rand_points, rand_queries
    import oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    pst = load_package()
    import importlib.util
    spec = importlib.util.spec_from_file_location("sharded", ROOT / "static-priority-search-tree_b200" / "sharded.py")
    sh = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(sh)
    torch.cuda.set_device(0)
    pts = rand_points(150001, dt, ids="random", dup=(dt == "i32"), seed=21)
    slab = sh.partition_by_dim1(pts, world)[rank]
    shard = sh.GpuShard(pst, pst.points_to_device(slab), len(slab), dt, True, max_queries=64)
    spst = sh.ShardedPST(shard)
    qs = rand_queries(pts, 100, seed=22)  # more than one engine batch per shard
    kinds = np.array([sh.QUERY_KINDS[k] for k, *_ in qs])
    t = oracle.DTYPES[dt]
    cols = [np.array([x[j] for x in qs], t) for j in (1, 2, 3)]
    res = spst.search(kinds, *cols, dst=0)
    ok = True
    if rank == 0:
        offs, recs = res
        ids = recs.numpy().view(np.uint32)
        full = oracle.Orc.build(pts, dt)
        for i, (kind, a, b, m2) in enumerate(qs):
            want = np.sort(oracle.Orc.search_ids(full, kind, a, b, m2))
            ok &= np.array_equal(np.sort(ids[int(offs[i]):int(offs[i + 1])]), want)
        q.put(bool(ok))
    shard.close()
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("dt", ["f32", "i32"])
def test_two_gpu_shards_equal_one_tree(dt):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q, dt)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert q.get(timeout=5) is True
