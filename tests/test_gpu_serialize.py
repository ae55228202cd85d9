"""Tree images (pst_save / pst_load and the file forms): a loaded tree is the saved
tree field for field (checked through pst_export against the oracle's build of
the same points) and answers every query identically; malformed images are
rejected with the documented status."""
import ctypes as C

import numpy as np
import pytest

from datagen import rand_points, rand_queries

pytestmark = pytest.mark.gpu

CASES = [("f32", "arange"), ("f64", "random"), ("i32", "desc"), ("f32", "none"), ("f64", "none")]


def _same_tree(a, b):
    ea, eb = a.export(), b.export()
    for k in ("dim1", "dim2", "med", "bitcodes"):
        assert ea[k].tobytes() == eb[k].tobytes(), k
    if ea["ids"] is not None:
        assert np.array_equal(ea["ids"], eb["ids"])


@pytest.mark.parametrize("dt,ids", CASES)
def test_image_round_trip(pst, oracle, tmp_path, dt, ids):
    pts = rand_points(70001, dt, ids=ids, dup=(dt == "i32"), seed=41)
    tree = pst.StaticPSTGPU.from_numpy(pts, dt)
    via_bytes = pst.StaticPSTGPU.from_bytes(tree.to_bytes())
    path = tmp_path / "tree.pstb"
    tree.save(path)
    via_file = pst.StaticPSTGPU.load(path)
    assert via_bytes.n == via_file.n == tree.n and via_bytes.dt == dt and via_bytes.has_id == tree.has_id
    _same_tree(tree, via_bytes)
    _same_tree(tree, via_file)
    ret = "ids" if tree.has_id else "points"
    for kind, a, b, c in rand_queries(pts, 12, seed=42):
        want = oracle.canon(tree.search(kind, a, b, c, ret=ret))
        assert np.array_equal(oracle.canon(via_bytes.search(kind, a, b, c, ret=ret)), want)
        assert np.array_equal(oracle.canon(via_file.search(kind, a, b, c, ret=ret)), want)
    for t in (tree, via_bytes, via_file):
        t.close()


def test_image_of_empty_and_tiny_trees(pst):
    for n in (0, 1, 2, 3):
        pts = rand_points(n, "f32", seed=43)
        tree = pst.StaticPSTGPU.from_numpy(pts, "f32")
        back = pst.StaticPSTGPU.from_bytes(tree.to_bytes())
        assert back.n == n
        if n:
            _same_tree(tree, back)
        tree.close()
        back.close()


def test_malformed_images_are_rejected(pst, tmp_path):
    tree = pst.StaticPSTGPU.from_numpy(rand_points(5000, "f32", seed=44), "f32")
    img = bytearray(tree.to_bytes())
    tree.close()
    INVALID, UNSUPPORTED = 1, 5
    bad_magic = bytes(b"XXXX" + img[4:])
    with pytest.raises(pst.PSTError) as e:
        pst.StaticPSTGPU.from_bytes(bad_magic)
    assert e.value.status == INVALID
    with pytest.raises(pst.PSTError) as e:
        pst.StaticPSTGPU.from_bytes(bytes(img[: len(img) // 2]))
    assert e.value.status == INVALID
    newer = bytearray(img)
    newer[8:12] = (99).to_bytes(4, "little")
    with pytest.raises(pst.PSTError) as e:
        pst.StaticPSTGPU.from_bytes(bytes(newer))
    assert e.value.status == UNSUPPORTED
    lied = bytearray(img)
    lied[24:32] = (123457).to_bytes(8, "little")  # point count that does not match the sizes
    with pytest.raises(pst.PSTError) as e:
        pst.StaticPSTGPU.from_bytes(bytes(lied))
    assert e.value.status == INVALID
    with pytest.raises(pst.PSTError) as e:
        pst.StaticPSTGPU.load(tmp_path / "missing.pstb")
    assert e.value.status == INVALID
    short = tmp_path / "short.pstb"
    short.write_bytes(bytes(img[:1000]))
    with pytest.raises(pst.PSTError) as e:
        pst.StaticPSTGPU.load(short)
    assert e.value.status == INVALID


def test_save_capacity(pst):
    tree = pst.StaticPSTGPU.from_numpy(rand_points(3000, "f32", seed=45), "f32")
    lib = pst.lib()
    need = C.c_uint64()
    assert lib.pst_image_size(tree.handle, C.byref(need)) == 0
    small = np.zeros(need.value - 1, np.uint8)
    written = C.c_uint64()
    st = lib.pst_save(tree.handle, small.ctypes.data_as(C.c_void_p), len(small), C.byref(written), None)
    assert st == 4 and written.value == need.value  # PST_ERR_CAPACITY, size still reported
    tree.close()
