"""pst_search_noalloc: the single-query search that allocates nothing (its working
memory is the library's static 8 MiB device array), for callers that cannot
allocate device memory while they search.  Checked through the C ABI against the
existing pst_search_into on the same tree and queries and against the CPU oracle,
two calls in a row each (the array keeps the previous call's contents, so the
second call checks that everything that must start at zero is reset)."""
import ctypes as C

import numpy as np
import pytest

from datagen import rand_points, rand_queries

pytestmark = pytest.mark.gpu

PST_OK, PST_ERR_CAPACITY = 0, 4


def _entry_points(pst):
    lib = pst.lib()
    Q = pst.pst.Query
    noalloc = lib.pst_search_noalloc
    noalloc.restype = C.c_int32
    noalloc.argtypes = [C.c_void_p, C.POINTER(Q), C.c_int32, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64),
                        C.c_void_p]
    into = lib.pst_search_into
    return noalloc, into


def _query(pst, dt, kind, a, b, c):
    v = pst.pst.value
    return pst.pst.Query(pst.pst.KIND[kind], 0, v(dt, a), v(dt, b), v(dt, c))


def _canon(oracle, raw, rec):
    return oracle.canon(raw.view(rec))


@pytest.mark.parametrize("dt", ["f32", "f64", "i32"])
def test_noalloc_equals_search_into(pst, oracle, dt):
    import torch
    pts = rand_points(300000, dt, ids="random", dup=(dt == "i32"), seed=31)
    tree = pst.StaticPSTGPU.from_numpy(pts, dt)
    noalloc, into = _entry_points(pst)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    n = len(pts)
    ref = oracle.Orc.build(pts, dt)
    for kind, a, b, m2 in rand_queries(pts, 6, seed=32):
        q = _query(pst, dt, kind, a, b, m2)
        expect = {"ids": oracle.canon(oracle.Orc.search_ids(ref, kind, a, b, m2)),
                  "points": oracle.canon(oracle.Orc.search_points(ref, kind, a, b, m2))}
        for ret, rec in (("ids", np.dtype(np.uint32)), ("points", pts.dtype)):
            rsz = rec.itemsize
            buf = torch.empty(n * rsz + 16, dtype=torch.uint8, device="cuda")
            cnt = C.c_uint64()
            assert into(tree.handle, C.byref(q), pst.pst.RET[ret], C.c_void_p(buf.data_ptr()), n, C.byref(cnt),
                        stream) == PST_OK
            want = _canon(oracle, buf[: cnt.value * rsz].cpu().numpy(), rec)
            assert np.array_equal(want, expect[ret]), (kind, ret)
            for _ in range(2):
                out = torch.full((n * rsz + 16,), 0xAB, dtype=torch.uint8, device="cuda")
                c2 = C.c_uint64()
                st = noalloc(tree.handle, C.byref(q), pst.pst.RET[ret], C.c_void_p(out.data_ptr()), n, C.byref(c2),
                             stream)
                assert st == PST_OK, pst.lib().pst_last_error()
                assert c2.value == cnt.value
                got = _canon(oracle, out[: c2.value * rsz].cpu().numpy(), rec)
                assert np.array_equal(got, want), (kind, ret)
    tree.close()


def test_noalloc_limits(pst):
    import torch
    noalloc, _ = _entry_points(pst)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    # output capacity: full count reported, nothing written
    pts = rand_points(100000, "f32", seed=33)
    tree = pst.StaticPSTGPU.from_numpy(pts, "f32")
    q = _query(pst, "f32", "left", 0, 800, 0)
    out = torch.zeros(16, dtype=torch.int32, device="cuda")
    cnt = C.c_uint64()
    assert noalloc(tree.handle, C.byref(q), 0, C.c_void_p(out.data_ptr()), 16, C.byref(cnt), stream) == PST_ERR_CAPACITY
    assert cnt.value > 16 and int(out.abs().sum().item()) == 0
    tree.close()
    # trees above the stated maximum (2^22 - 1 points) are rejected up front
    big = pst.StaticPSTGPU.from_numpy(rand_points(1 << 22, "f32", seed=34), "f32")
    assert noalloc(big.handle, C.byref(q), 0, C.c_void_p(out.data_ptr()), 16, C.byref(cnt), stream) == PST_ERR_CAPACITY
    assert b"4194303" in pst.lib().pst_last_error()
    big.close()
