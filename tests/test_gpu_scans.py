"""GPU parity of the streaming kernels: interval parallel search and metacells."""
import numpy as np
import pytest

from datagen import rand_points

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dt", ["f32", "f64", "i32"])
@pytest.mark.parametrize("ids", ["arange", "random", "none"])
def test_ips(pst, oracle, dt, ids):
    pts = rand_points(123457, dt, ids=ids, dup=(dt == "i32"), seed=7)
    d = pst.points_to_device(pts)
    for v in [pts["dim1"][5], pts["dim2"][77], 500, -1e9 if dt != "i32" else -10**9]:
        idx = oracle.Orc.ips(pts, dt, v)
        if ids != "none":
            got = pst.intervalParallelSearch(d, len(pts), v, dt, True, ret="ids")
            assert np.array_equal(np.sort(got), np.sort(pts["id"][idx]))
        gotp = pst.intervalParallelSearch(d, len(pts), v, dt, ids != "none", ret="points")
        assert np.array_equal(oracle.canon(gotp), oracle.canon(pts[idx]))


def test_ips_equals_pst_left(pst, oracle):
    """IPS(v) is the 2-sided-left query (v, v)."""
    pts = rand_points(200000, "f32", ids="arange", seed=12)
    d = pst.points_to_device(pts)
    tr = pst.StaticPSTGPU(d, len(pts), "f32", True)
    for v in [100.0, 333.25, 999.0]:
        a = pst.intervalParallelSearch(d, len(pts), v, "f32", True)
        b = tr.twoSidedLeftSearch(v, v, ret="ids")
        assert np.array_equal(np.sort(a), np.sort(b))
    tr.close()


@pytest.mark.parametrize("dims,mc", [((17, 13, 9), (4, 4, 4)), ((33, 33, 33), (4, 4, 4)), ((20, 7, 11), (3, 2, 5)),
                                     ((9, 10, 11), (1, 1, 1)), ((66, 40, 35), (4, 4, 4)), ((2, 2, 2), (4, 4, 4))])
@pytest.mark.parametrize("dt", ["f32", "f64"])
def test_metacells(pst, oracle, dims, mc, dt):
    import torch
    rng = np.random.default_rng(sum(dims))
    px, py, pz = dims
    vol = rng.standard_normal((pz, py, px)).astype(np.float32 if dt == "f32" else np.float64)
    lo, hi, ids = oracle.Orc.metacells(vol, dt, dims, mc)
    vd = torch.from_numpy(vol.reshape(-1).copy()).to("cuda")
    out, n = pst.formMetacellTags(vd, dims, mc, dt, True)
    rec = out.cpu().numpy().view(pst.point_dtype(dt, True))
    assert n == len(lo)
    assert rec["dim1"].tobytes() == lo.tobytes()
    assert rec["dim2"].tobytes() == hi.tobytes()
    assert np.array_equal(rec["id"], ids)
    out2, _ = pst.formMetacellTags(vd, dims, mc, dt, False)
    rec2 = out2.cpu().numpy().view(pst.point_dtype(dt, False))
    assert rec2["dim1"].tobytes() == lo.tobytes() and rec2["dim2"].tobytes() == hi.tobytes()


@pytest.mark.parametrize("dims,mc", [((64, 13, 9), (4, 4, 4)), ((36, 33, 17), (4, 4, 4)), ((4, 4, 4), (4, 4, 4)),
                                     ((8, 5, 6), (4, 2, 3)), ((1028, 3, 3), (4, 4, 4)), ((16, 9, 2), (4, 4, 1))])
@pytest.mark.parametrize("dt", ["f32", "i32", "f64"])
@pytest.mark.parametrize("zeros", [False, True])
def test_metacells_aligned_rows(pst, oracle, dims, mc, dt, zeros):
    """Rows a multiple of 4 vertices long under 4-wide metacells (the layout whose rows
    are read 16 bytes at a time for 4-byte values): ragged last metacells, rows wider
    than one CTA, and (zeros) volumes of -0.0 / +0.0 / +-1 / 2, whose min and max
    must keep the same zero as the CPU restatement, bit for bit."""
    import torch
    rng = np.random.default_rng(sum(dims) + 3)
    px, py, pz = dims
    npdt = {"f32": np.float32, "f64": np.float64, "i32": np.int32}[dt]
    if zeros and dt != "i32":
        vol = rng.choice(np.array([-0.0, 0.0, -1.0, 1.0, 2.0], npdt), (pz, py, px))
    elif dt == "i32":
        vol = rng.integers(-50, 50, (pz, py, px)).astype(np.int32)
    else:
        vol = rng.standard_normal((pz, py, px)).astype(npdt)
    lo, hi, ids = oracle.Orc.metacells(vol, dt, dims, mc)
    vd = torch.from_numpy(vol.reshape(-1).copy()).to("cuda")
    out, n = pst.formMetacellTags(vd, dims, mc, dt, True)
    rec = out.cpu().numpy().view(pst.point_dtype(dt, True))
    assert n == len(lo)
    assert rec["dim1"].tobytes() == lo.tobytes()
    assert rec["dim2"].tobytes() == hi.tobytes()
    assert np.array_equal(rec["id"], ids)


@pytest.mark.parametrize("dt", ["f32", "i32", "f64"])
def test_ips_unaligned_points(pst, oracle, dt):
    """A point array that starts one record into its allocation (not on a 16-byte
    boundary) is scanned without the 16-byte staging; the results are the same."""
    pts = rand_points(50001, dt, ids="arange", dup=(dt == "i32"), seed=9)
    d = pst.points_to_device(pts)
    sub = pts[1:]
    dv = d[pts.dtype.itemsize:]
    for v in [sub["dim1"][3], sub["dim2"][100], sub["dim1"][-1]]:
        idx = oracle.Orc.ips(sub, dt, v)
        got = pst.intervalParallelSearch(dv, len(sub), v, dt, True, ret="ids")
        assert np.array_equal(np.sort(got), np.sort(sub["id"][idx]))
        gotp = pst.intervalParallelSearch(dv, len(sub), v, dt, True, ret="points")
        assert np.array_equal(oracle.canon(gotp), oracle.canon(sub[idx]))


@pytest.mark.parametrize("dt", ["f32", "i32"])
def test_metacells_unaligned_volume(pst, oracle, dt):
    """A volume that starts one value into its allocation (not on a 16-byte
    boundary) is reduced without the 16-byte row loads; the records are the same."""
    import torch
    dims, mc = (64, 9, 7), (4, 4, 4)
    rng = np.random.default_rng(77)
    px, py, pz = dims
    if dt == "i32":
        vol = rng.integers(-99, 99, (pz, py, px)).astype(np.int32)
    else:
        vol = rng.standard_normal((pz, py, px)).astype(np.float32)
    lo, hi, ids = oracle.Orc.metacells(vol, dt, dims, mc)
    big = np.concatenate([np.zeros(1, vol.dtype), vol.reshape(-1)])
    vd = torch.from_numpy(big).to("cuda")[1:]
    out, n = pst.formMetacellTags(vd, dims, mc, dt, True)
    rec = out.cpu().numpy().view(pst.point_dtype(dt, True))
    assert n == len(lo)
    assert rec["dim1"].tobytes() == lo.tobytes() and rec["dim2"].tobytes() == hi.tobytes()
    assert np.array_equal(rec["id"], ids)
