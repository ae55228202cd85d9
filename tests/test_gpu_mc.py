"""Marching cubes over active metacells (pst_mc_count / pst_mc_triangles): the
triangles equal the CPU restatement's bit for bit and in order; the metacells the
PST reports for (iso, iso) carry every triangle of the isosurface (the other
metacells have none); the surface is closed and consistently oriented."""
import sys
from pathlib import Path

import numpy as np
import pytest

from datagen import blob_volume

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import marching_cubes as mc  # noqa: E402

pytestmark = pytest.mark.gpu


def _grid(dims, mcd):
    return [-(-(dims[i] - 1) // mcd[i]) for i in range(3)]


@pytest.mark.parametrize("dims,mcd,iso", [
    ((17, 13, 11), (4, 4, 4), 0.5),
    ((18, 14, 10), (4, 4, 4), 0.3),   # ragged last metacells
    ((9, 10, 12), (2, 3, 5), 0.7),
    ((8, 8, 8), (1, 1, 1), 0.5),      # one cell per metacell
    ((21, 14, 13), (8, 4, 4), 0.4),   # metacells of more vertices than a warp holds in registers
])
def test_random_volume_equals_cpu(pst, dims, mcd, iso):
    import torch
    rng = np.random.default_rng(61)
    vol = rng.random(dims[::-1]).astype(np.float32)
    M = _grid(dims, mcd)
    ids = np.arange(M[0] * M[1] * M[2], dtype=np.uint32)
    rng.shuffle(ids)  # output follows the given order
    want = mc.metacell_triangles(vol, mcd, ids, iso)
    vd = torch.from_numpy(vol.reshape(-1)).to("cuda")
    got = pst.marchingCubes(vd, dims, mcd, torch.from_numpy(ids).to("cuda"), iso).cpu().numpy()
    assert got.shape == want.shape
    assert got.tobytes() == want.tobytes()


def test_isosurface_from_active_metacells(pst, oracle):
    import torch
    dims = (96, 80, 72)
    vol = blob_volume(*dims, nblobs=8, sigma=(4.0, 12.0), seed=62)
    vd = torch.from_numpy(vol.reshape(-1)).to("cuda")
    recs, n = pst.formMetacellTags(vd, dims, (4, 4, 4), "f32", True)
    tree = pst.StaticPSTGPU(recs, n, "f32", True)
    all_ids = torch.arange(n, dtype=torch.int32, device="cuda")
    for iso in (0.15, 0.4):
        act = np.sort(tree.twoSidedLeftSearch(np.float32(iso), np.float32(iso), ret="ids")).astype(np.uint32)
        act_d = torch.from_numpy(act).to("cuda")
        got = pst.marchingCubes(vd, dims, (4, 4, 4), act_d, iso).cpu().numpy()
        want = mc.metacell_triangles(vol, (4, 4, 4), act, iso)
        assert got.tobytes() == want.tobytes(), iso
        # the whole volume gives the same triangles: inactive metacells contribute none
        every = pst.marchingCubes(vd, dims, (4, 4, 4), all_ids, iso).cpu().numpy()
        assert np.array_equal(np.sort(every.view(np.uint32).reshape(-1, 9), axis=0),
                              np.sort(got.view(np.uint32).reshape(-1, 9), axis=0))
        assert len(got) > 1000
        assert mc.mesh_defects(got, dims) == (0, 0)
    tree.close()


def test_limits(pst):
    import torch
    import ctypes as C
    vol = torch.rand(10 * 10 * 10, device="cuda")
    ids = torch.arange(27, dtype=torch.int32, device="cuda")
    assert pst.marchingCubes(vol, (10, 10, 10), (4, 4, 4), ids[:0], 0.5).shape[0] == 0
    lib = pst.lib()
    P = (C.c_uint32 * 3)(10, 10, 10)
    M = (C.c_uint32 * 3)(4, 4, 4)
    cnt, got = C.c_uint64(), C.c_uint64()
    assert lib.pst_mc_count(C.c_void_p(vol.data_ptr()), P, M, C.c_void_p(ids.data_ptr()), 27, C.c_float(0.5),
                            C.byref(cnt), None) == 0
    assert cnt.value > 1
    small = torch.empty((1, 9), device="cuda")
    st = lib.pst_mc_triangles(C.c_void_p(vol.data_ptr()), P, M, C.c_void_p(ids.data_ptr()), 27, C.c_float(0.5),
                              C.c_void_p(small.data_ptr()), 1, C.byref(got), None)
    assert st == 4 and got.value == cnt.value  # PST_ERR_CAPACITY, full count reported
