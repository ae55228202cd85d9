"""Isosurface active-metacell path: a 512^3 float32 volume of 32 Gaussian blobs plus
N(0, 0.01) noise; 4^3-voxel metacells sharing boundary vertices (128^3 points);
twoSidedLeftSearch(iso, iso) at 16 isovalues 0.05 + 0.06 i, against the interval
parallel search and the oracle."""
import numpy as np
import pytest

from datagen import blob_volume

pytestmark = pytest.mark.gpu


def test_isosurface_512(pst, oracle):
    import torch
    dims = (512, 512, 512)
    vol = blob_volume(*dims, seed=1)
    lo, hi, ids = oracle.Orc.metacells(vol, "f32", dims, (4, 4, 4))
    vd = torch.from_numpy(vol.reshape(-1)).to("cuda")
    mc_d, n = pst.formMetacellTags(vd, dims, (4, 4, 4), "f32", True)
    assert n == 128 ** 3
    rec = mc_d.cpu().numpy().view(pst.point_dtype("f32", True))
    assert rec["dim1"].tobytes() == lo.tobytes() and rec["dim2"].tobytes() == hi.tobytes()
    assert np.array_equal(rec["id"], ids)
    tree = pst.StaticPSTGPU(mc_d, n, "f32", True)
    ref = oracle.Orc.build(rec, "f32")
    for i in range(16):
        iso = np.float32(0.05 + 0.06 * i)
        got = tree.twoSidedLeftSearch(iso, iso, ret="ids")
        ips = pst.intervalParallelSearch(mc_d, n, iso, "f32", True, ret="ids")
        want = oracle.Orc.search_ids(ref, "left", 0, iso, iso)
        assert np.array_equal(np.sort(got), np.sort(want)), i
        assert np.array_equal(np.sort(ips), np.sort(want)), i
    tree.close()
