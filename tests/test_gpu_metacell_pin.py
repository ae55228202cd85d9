"""The metacell oracle pinned to the reference itself: the reference's own
formMetacellTags kernel (helpers/isosurface-data-processing.h:69-137,
helpers/isosurface-data-processing.tu:9-127, :181-212), compiled from its sources
by oracle/Makefile into oracle/_ref/libmcref.so, run on the GPU over seeded
volumes, and compared record for record with the oracle's restatement
(Orc.metacells) and with this library's pst_form_metacells.

Only sizes the reference's kernel handles are run: (P - 1) mod mc != 0 on every
axis (its grid-stride loops then run once) and every warp's first thread on a valid
voxel of the last metacell of each axis; the harness refuses other sizes without
launching anything."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from datagen import blob_volume

pytestmark = pytest.mark.gpu

REF_MC = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "libmcref.so"
DT_CODE = {"f32": 0, "f64": 1, "i32": 2}
NP_T = {"f32": np.float32, "f64": np.float64, "i32": np.int32}


def _lib():
    if not REF_MC.exists():
        pytest.skip("oracle/_ref/libmcref.so was not built (the reference sources were absent)")
    lib = C.CDLL(str(REF_MC))
    lib.ref_metacells.restype = C.c_int64
    lib.ref_metacells.argtypes = [C.c_int, C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.c_void_p]
    return lib


def _volume(dims, dt, seed):
    px, py, pz = dims
    vol = blob_volume(px, py, pz, nblobs=6, seed=seed, sigma=(2.0, 8.0))
    if dt == "i32":
        return np.round(vol * 1000).astype(np.int32)
    return vol.astype(NP_T[dt])


# 4^3 metacells: two warps, the second starting at z = 2, so (P_z - 1) mod 4 == 3;
# 2^3 and 8x2x2: one warp; 2x4x8: the second warp starts at z = 4.
CASES = [("f32", (8, 8, 8), (4, 4, 4)), ("f32", (64, 50, 40), (4, 4, 4)), ("f32", (102, 35, 12), (4, 4, 4)),
         ("f32", (10, 6, 8), (2, 2, 2)), ("f32", (19, 8, 10), (8, 2, 2)), ("f32", (12, 14, 15), (2, 4, 8)),
         ("f64", (64, 50, 40), (4, 4, 4)), ("i32", (64, 48, 40), (4, 4, 4)), ("i32", (27, 12, 14), (8, 2, 2))]


@pytest.mark.parametrize("dt,dims,mc", CASES)
def test_reference_metacells_equal_oracle_and_library(pst, oracle, dt, dims, mc):
    import torch
    lib = _lib()
    vol = _volume(dims, dt, seed=sum(dims))
    lo, hi, ids = oracle.Orc.metacells(vol, dt, dims, mc)
    n = len(lo)
    rec = oracle.point_dtype(dt, True)
    vol_d = torch.from_numpy(vol.reshape(-1).copy()).to("cuda")
    out_d = torch.zeros(n * rec.itemsize, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    P = (C.c_uint32 * 3)(*dims)
    M = (C.c_uint32 * 3)(*mc)
    got_n = lib.ref_metacells(DT_CODE[dt], C.c_void_p(vol_d.data_ptr()), P, M, C.c_void_p(out_d.data_ptr()))
    assert got_n == n
    ref = out_d.cpu().numpy().view(rec)
    # the reference's records, bit for bit, against the oracle's restatement
    assert ref["dim1"].tobytes() == lo.tobytes()
    assert ref["dim2"].tobytes() == hi.tobytes()
    assert np.array_equal(ref["id"], ids)
    # and against this library's metacell kernel
    mine, n2 = pst.formMetacellTags(vol_d, dims, mc, dt, True)
    assert n2 == n
    got = mine.cpu().numpy().view(rec)
    # field by field: the reference leaves the records' padding bytes as they were
    for f in ("dim1", "dim2", "id"):
        assert got[f].tobytes() == ref[f].tobytes(), f


def test_reference_harness_refuses_sizes_it_mishandles():
    """(P - 1) divisible by mc would make the reference's loops run a second pass that
    writes past the metacell grid: the harness returns -1 and launches nothing."""
    lib = _lib()
    P = (C.c_uint32 * 3)(9, 9, 9)
    M = (C.c_uint32 * 3)(4, 4, 4)
    assert lib.ref_metacells(0, None, P, M, None) == -1
    P2 = (C.c_uint32 * 3)(8, 8, 11)  # the second warp's first thread (z = 2) has no voxel in the last z-metacell
    assert lib.ref_metacells(0, None, P2, M, None) == -1
