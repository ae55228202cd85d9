"""Volume ingest: raw volume files read straight into device memory
(pst_read_volume, the reference's readInVertices) and metacell formation streamed
from the file in z-slabs (pst_form_metacells_from_file), which must give the same
records, bit for bit, as pst_form_metacells over the whole volume on the device;
missing and short files are PST_ERR_INVALID (the reference exits)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NP = {"f32": np.float32, "f64": np.float64, "i32": np.int32}


def _volume(dims, dt, seed):
    rng = np.random.default_rng(seed)
    px, py, pz = dims
    if dt == "i32":
        return rng.integers(-1000, 1000, (pz, py, px)).astype(np.int32)
    return (rng.standard_normal((pz, py, px)) * 10).astype(NP[dt])


@pytest.mark.parametrize("dt", ["f32", "f64", "i32"])
def test_read_volume(pst, tmp_path, dt):
    import torch
    vol = _volume((37, 21, 13), dt, 51)
    path = tmp_path / "vol.raw"
    vol.tofile(path)
    d = pst.readInVertices(path, vol.size, dt)
    assert np.array_equal(d.cpu().numpy(), vol.reshape(-1))
    # a prefix of a longer file, as the reference reads exactly num_vertices values
    d2 = pst.readInVertices(path, vol.size - 100, dt)
    assert np.array_equal(d2.cpu().numpy(), vol.reshape(-1)[: vol.size - 100])
    torch.cuda.synchronize()


@pytest.mark.parametrize("dt,dims,mc,slab", [
    ("f32", (65, 33, 41), (4, 4, 4), 0),          # one slab
    ("f32", (65, 33, 41), (4, 4, 4), 1),          # one metacell layer per slab
    ("f32", (66, 35, 42), (4, 4, 4), 20000),      # ragged last metacells, several layers per slab
    ("f64", (30, 17, 29), (3, 2, 5), 9000),
    ("i32", (19, 23, 31), (2, 3, 4), 1),
    ("f32", (9, 9, 9), (1, 1, 1), 500),           # voxel tags
])
def test_metacells_from_file_equal_whole_volume(pst, tmp_path, dt, dims, mc, slab):
    import torch
    vol = _volume(dims, dt, 52)
    path = tmp_path / "vol.raw"
    vol.tofile(path)
    for has_id in (True, False):
        dev = torch.from_numpy(vol.reshape(-1).copy()).to("cuda")
        want, n = pst.formMetacellTags(dev, dims, mc, dt, has_id)
        got, n2 = pst.formMetacellTagsFromFile(path, dims, mc, dt, has_id, slab_bytes=slab)
        assert n == n2
        rec = pst.point_dtype(dt, has_id)
        w, g = want.cpu().numpy().view(rec), got.cpu().numpy().view(rec)
        for f in rec.names:  # field by field: the padding bytes of f64 records are unset
            assert w[f].tobytes() == g[f].tobytes(), f


def test_ingest_errors(pst, tmp_path):
    vol = _volume((8, 8, 8), "f32", 53)
    path = tmp_path / "vol.raw"
    vol.tofile(path)
    INVALID = 1
    with pytest.raises(pst.PSTError) as e:
        pst.readInVertices(tmp_path / "missing.raw", 10, "f32")
    assert e.value.status == INVALID
    with pytest.raises(pst.PSTError) as e:
        pst.readInVertices(path, vol.size + 1, "f32")
    assert e.value.status == INVALID
    with pytest.raises(pst.PSTError) as e:
        pst.formMetacellTagsFromFile(path, (8, 8, 9), (4, 4, 4), "f32")
    assert e.value.status == INVALID
