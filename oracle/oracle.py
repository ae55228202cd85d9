"""ctypes front end of the CPU oracle.  TEST INFRASTRUCTURE ONLY.

Two back ends, both CPU:

* ``Orc``  - liborc.so, the plain-C restatement in pst_oracle.c (always built).
* ``Ref``  - _ref/libpstref.so, the reference's own StaticPSTCPUIter compiled
  unmodified from its sources by the Makefile here (built only where the
  reference sources exist; the built file travels with the repository copy).

Only the tests, the smoke check and the CPU-baseline leg of the benchmark use
this module, always as the checker, never as the thing measured for the GPU
path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORC_SO = HERE / "liborc.so"
REF_SO = HERE / "_ref" / "libpstref.so"

DTYPES = {"f32": np.float32, "f64": np.float64, "i32": np.int32}
DTYPE_CODE = {"f32": 0, "f64": 1, "i32": 2}
Q_THREE, Q_LEFT, Q_RIGHT = 0, 1, 2
KINDS = {"three": Q_THREE, "left": Q_LEFT, "right": Q_RIGHT}


def point_dtype(dt: str, has_id: bool) -> np.dtype:
    """numpy view of the reference's PointStruct<T, uint32_t, 1> / <T, void, 0>
    (helpers/point-struct.h:25-33, :106-117), with C alignment and padding."""
    t = DTYPES[dt]
    fields = [("dim1", t), ("dim2", t)]
    if has_id:
        fields.append(("id", np.uint32))
    return np.dtype(fields, align=True)


def make_points(dim1, dim2, ids=None, dt: str = "f32") -> np.ndarray:
    pts = np.zeros(len(dim1), dtype=point_dtype(dt, ids is not None))
    pts["dim1"] = dim1
    pts["dim2"] = dim2
    if ids is not None:
        pts["id"] = ids
    return pts


def num_slots(n: int) -> int:
    return 0 if n == 0 else (1 << int(n).bit_length()) - 1


def build_oracle_libs(ref_root: str | None = None) -> None:
    """Compile liborc.so (and _ref/libpstref.so where the reference exists)."""
    env = dict(os.environ)
    if ref_root:
        env["REF_ROOT"] = ref_root
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True, env=env)


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Tree:
    """Tree in the reference's field layout (heap slot s, root 0)."""

    def __init__(self, dt: str, has_id: bool, n: int):
        S = num_slots(n)
        t = DTYPES[dt]
        self.dt, self.has_id, self.n, self.S = dt, has_id, n, S
        self.dim1 = np.zeros(S, t)
        self.dim2 = np.zeros(S, t)
        self.med = np.zeros(S, t)
        self.ids = np.zeros(S, np.uint32) if has_id else None
        self.bitcodes = np.zeros(S, np.uint8)

    def equal(self, other: "Tree") -> bool:
        same = (self.S == other.S
                and self.dim1.tobytes() == other.dim1.tobytes()
                and self.dim2.tobytes() == other.dim2.tobytes()
                and self.med.tobytes() == other.med.tobytes()
                and self.bitcodes.tobytes() == other.bitcodes.tobytes())
        if self.has_id:
            same = same and self.ids.tobytes() == other.ids.tobytes()
        return same


class Orc:
    """The C restatement (pst_oracle.c)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not ORC_SO.exists():
                build_oracle_libs()
            lib = C.CDLL(str(ORC_SO))
            for sfx, ct in (("f32", C.c_float), ("f64", C.c_double), ("i32", C.c_int32)):
                f = getattr(lib, f"orc_build_{sfx}")
                f.restype = C.c_int
                f.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_int, C.c_uint64] + [C.c_void_p] * 5
                f = getattr(lib, f"orc_search_{sfx}")
                f.restype = C.c_int64
                f.argtypes = [C.c_void_p] * 4 + [C.c_uint64, C.c_int, ct, ct, ct, C.c_void_p]
                f = getattr(lib, f"orc_brute_{sfx}")
                f.restype = C.c_int64
                f.argtypes = [C.c_void_p, C.c_size_t, C.c_uint64, C.c_int, ct, ct, ct, C.c_void_p]
                f = getattr(lib, f"orc_ips_{sfx}")
                f.restype = C.c_int64
                f.argtypes = [C.c_void_p, C.c_size_t, C.c_uint64, ct, C.c_void_p]
                f = getattr(lib, f"orc_brute_multi_{sfx}")
                f.restype = C.c_int64
                f.argtypes = [C.c_void_p, C.c_size_t, C.c_uint64, C.c_uint32] + [C.c_void_p] * 4 + \
                    [C.c_int, C.c_void_p, C.c_void_p]
                f = getattr(lib, f"orc_metacells_{sfx}")
                f.restype = C.c_int64
                f.argtypes = [C.c_void_p] + [C.c_uint32] * 6 + [C.c_void_p] * 3
            cls._lib = lib
        return cls._lib

    @classmethod
    def build(cls, pts: np.ndarray, dt: str) -> Tree:
        has_id = "id" in pts.dtype.names
        pts = np.ascontiguousarray(pts)
        tr = Tree(dt, has_id, len(pts))
        off = pts.dtype.fields["id"][1] if has_id else 0
        rc = getattr(cls.lib(), f"orc_build_{dt}")(
            _ptr(pts), pts.dtype.itemsize, off, int(has_id), len(pts),
            _ptr(tr.dim1), _ptr(tr.dim2), _ptr(tr.med), _ptr(tr.ids), _ptr(tr.bitcodes))
        if rc != 0:
            raise RuntimeError(f"oracle build failed ({rc})")
        return tr

    @classmethod
    def search_slots(cls, tr: Tree, kind: str, min1=0, max1=0, min2=0) -> np.ndarray:
        out = np.zeros(max(tr.n, 1), np.uint64)
        cnt = getattr(cls.lib(), f"orc_search_{tr.dt}")(
            _ptr(tr.dim1), _ptr(tr.dim2), _ptr(tr.med), _ptr(tr.bitcodes), tr.n,
            KINDS[kind], min1, max1, min2, _ptr(out))
        if cnt < 0:
            raise RuntimeError("oracle search failed")
        return out[:cnt]

    @classmethod
    def search_ids(cls, tr: Tree, kind: str, min1=0, max1=0, min2=0) -> np.ndarray:
        return tr.ids[cls.search_slots(tr, kind, min1, max1, min2)]

    @classmethod
    def search_points(cls, tr: Tree, kind: str, min1=0, max1=0, min2=0) -> np.ndarray:
        s = cls.search_slots(tr, kind, min1, max1, min2)
        res = np.zeros(len(s), point_dtype(tr.dt, tr.has_id))
        res["dim1"], res["dim2"] = tr.dim1[s], tr.dim2[s]
        if tr.has_id:
            res["id"] = tr.ids[s]
        return res

    @classmethod
    def brute(cls, pts: np.ndarray, dt: str, kind: str, min1=0, max1=0, min2=0) -> np.ndarray:
        pts = np.ascontiguousarray(pts)
        out = np.zeros(max(len(pts), 1), np.uint64)
        cnt = getattr(cls.lib(), f"orc_brute_{dt}")(
            _ptr(pts), pts.dtype.itemsize, len(pts), KINDS[kind], min1, max1, min2, _ptr(out))
        return out[:cnt]

    @classmethod
    def brute_multi(cls, pts: np.ndarray, dt: str, kinds, min1, max1, min2, threads: int | None = None,
                    counts_only: bool = False):
        """Brute force of many queries in one threaded pass over the points (for large
        point sets): returns (offsets[nq + 1], input indices), each query's indices in
        index order (only the offsets, and no indices, with counts_only)."""
        pts = np.ascontiguousarray(pts)
        t = DTYPES[dt]
        k = np.ascontiguousarray(np.asarray(kinds, np.int32))
        a, b, c = (np.ascontiguousarray(np.asarray(x, t)) for x in (min1, max1, min2))
        nq = len(k)
        th = threads or os.cpu_count() or 1
        off = np.zeros(nq + 1, np.uint64)
        fn = getattr(cls.lib(), f"orc_brute_multi_{dt}")
        tot = fn(_ptr(pts), pts.dtype.itemsize, len(pts), nq, _ptr(k), _ptr(a), _ptr(b), _ptr(c), th, _ptr(off),
                 None)
        if tot < 0:
            raise RuntimeError("oracle brute_multi failed")
        if counts_only:
            return off, None
        idx = np.zeros(max(int(tot), 1), np.uint64)
        tot2 = fn(_ptr(pts), pts.dtype.itemsize, len(pts), nq, _ptr(k), _ptr(a), _ptr(b), _ptr(c), th, _ptr(off),
                  _ptr(idx))
        if tot2 != tot:
            raise RuntimeError("oracle brute_multi failed")
        return off, idx[:tot]

    @classmethod
    def ips(cls, pts: np.ndarray, dt: str, v) -> np.ndarray:
        pts = np.ascontiguousarray(pts)
        out = np.zeros(max(len(pts), 1), np.uint64)
        cnt = getattr(cls.lib(), f"orc_ips_{dt}")(_ptr(pts), pts.dtype.itemsize, len(pts), v, _ptr(out))
        return out[:cnt]

    @classmethod
    def metacells(cls, vol: np.ndarray, dt: str, dims, mc=(4, 4, 4)):
        """vol is x-fastest with shape (pz, py, px); returns (min, max, id) arrays."""
        px, py, pz = dims
        M = [(p - 1 + m - 1) // m for p, m in zip(dims, mc)]
        n = M[0] * M[1] * M[2]
        lo = np.zeros(n, DTYPES[dt])
        hi = np.zeros(n, DTYPES[dt])
        ids = np.zeros(n, np.uint32)
        vol = np.ascontiguousarray(vol, dtype=DTYPES[dt])
        cnt = getattr(cls.lib(), f"orc_metacells_{dt}")(
            _ptr(vol), px, py, pz, mc[0], mc[1], mc[2], _ptr(lo), _ptr(hi), _ptr(ids))
        assert cnt == n
        return lo, hi, ids


class Ref:
    """The reference's StaticPSTCPUIter (or, with recursive=True, its
    StaticPSTCPURecur: searches only) compiled from its own sources."""

    _lib = None

    @classmethod
    def available(cls) -> bool:
        return REF_SO.exists()

    @classmethod
    def lib(cls):
        if cls._lib is None:
            lib = C.CDLL(str(REF_SO))
            lib.ref_build.restype = C.c_void_p
            lib.ref_build.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_uint64]
            lib.ref_build_recur.restype = C.c_void_p
            lib.ref_build_recur.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_uint64]
            lib.ref_destroy.argtypes = [C.c_void_p]
            lib.ref_num_slots.restype = C.c_uint64
            lib.ref_num_slots.argtypes = [C.c_void_p]
            lib.ref_export.argtypes = [C.c_void_p] * 6
            lib.ref_search.restype = C.c_int64
            lib.ref_search.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_int, C.c_void_p, C.c_uint64]
            cls._lib = lib
        return cls._lib

    def __init__(self, pts: np.ndarray, dt: str, recursive: bool = False):
        self.pts = np.ascontiguousarray(pts)
        self.dt = dt
        self.has_id = "id" in pts.dtype.names
        self.n = len(pts)
        self.recursive = recursive
        build = self.lib().ref_build_recur if recursive else self.lib().ref_build
        self.h = build(DTYPE_CODE[dt], int(self.has_id), _ptr(self.pts), self.n)
        if not self.h:
            raise RuntimeError("reference build failed")

    def close(self):
        if self.h:
            self.lib().ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def export(self) -> Tree:
        tr = Tree(self.dt, self.has_id, self.n)
        assert self.lib().ref_num_slots(self.h) == tr.S
        self.lib().ref_export(self.h, _ptr(tr.dim1), _ptr(tr.dim2), _ptr(tr.med), _ptr(tr.ids),
                              _ptr(tr.bitcodes))
        return tr

    def _bounds(self, min1, max1, min2):
        t = DTYPES[self.dt]
        return [np.array([v], t) for v in (min1, max1, min2)]

    def search(self, kind: str, min1=0, max1=0, min2=0, points: bool = False) -> np.ndarray:
        b = self._bounds(min1, max1, min2)
        rt = point_dtype(self.dt, self.has_id) if (points or not self.has_id) else np.uint32
        out = np.zeros(max(self.n, 1), rt)
        cnt = self.lib().ref_search(self.h, KINDS[kind], _ptr(b[0]), _ptr(b[1]), _ptr(b[2]),
                                    int(points or not self.has_id), _ptr(out), len(out))
        if cnt < 0:
            raise RuntimeError("reference search failed")
        return out[:cnt]

    def count(self, kind: str, min1=0, max1=0, min2=0) -> int:
        """Runs a search for its count only (results are discarded)."""
        b = self._bounds(min1, max1, min2)
        cnt = self.lib().ref_search(self.h, KINDS[kind], _ptr(b[0]), _ptr(b[1]), _ptr(b[2]),
                                    int(not self.has_id), None, 0)
        if cnt < 0:
            raise RuntimeError("reference search failed")
        return cnt


def canon(points_or_ids: np.ndarray) -> np.ndarray:
    """Order-independent canonical form of a result set for exact comparison.

    Ids sort as integers.  Point records compare by their fields' bit patterns
    (padding excluded), so -0.0 and +0.0 stay distinct, as stored."""
    a = np.asarray(points_or_ids)
    if a.dtype.names is None:
        return np.sort(a.astype(np.uint64))
    cols = [a["dim1"].view(f"u{a['dim1'].itemsize}").astype(np.uint64),
            a["dim2"].view(f"u{a['dim2'].itemsize}").astype(np.uint64)]
    if "id" in a.dtype.names:
        cols.append(a["id"].astype(np.uint64))
    rec = np.stack(cols, axis=1) if cols else np.zeros((0, 2), np.uint64)
    order = np.lexsort(rec.T[::-1])
    return rec[order]
