"""ctypes binding of libpst_b200.so (include/pst_c.h) with the reference's API shape."""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
library_path = _PKG / "libpst_b200.so"

DTYPE = {"f32": 0, "f64": 1, "i32": 2}
NP = {"f32": np.float32, "f64": np.float64, "i32": np.int32}
IDTYPE = {False: 0, True: 1}
RET = {"ids": 0, "points": 1}
KIND = {"three": 0, "left": 1, "right": 2}
STATUS = {0: "PST_OK", 1: "PST_ERR_INVALID", 2: "PST_ERR_CUDA", 3: "PST_ERR_NOMEM", 4: "PST_ERR_CAPACITY",
          5: "PST_ERR_UNSUPPORTED", 6: "PST_ERR_INTERNAL", 7: "PST_ERR_BUSY", 8: "PST_ERR_TIMEOUT"}


class PSTError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class Value(C.Union):
    _fields_ = [("f32", C.c_float), ("f64", C.c_double), ("i32", C.c_int32)]


class Query(C.Structure):
    _fields_ = [("kind", C.c_int32), ("reserved", C.c_int32), ("min1", Value), ("max1", Value), ("min2", Value)]


class BatchOpts(C.Structure):
    _fields_ = [("max_queries", C.c_uint32), ("task_capacity", C.c_uint64), ("block_threads", C.c_uint32),
                ("blocks_per_sm", C.c_uint32), ("use_graph", C.c_int32), ("emit_records", C.c_uint32),
                ("top_pass_queries", C.c_uint32)]


# The launch-shape fields of BatchOpts a tuning (the autotuner's choice) sets.
TUNING_FIELDS = ("block_threads", "blocks_per_sm", "emit_records", "top_pass_queries")


class ServerOpts(C.Structure):
    _fields_ = [("max_batch", C.c_uint32), ("slots_per_tree", C.c_uint32), ("out_budget_bytes", C.c_uint64),
                ("use_graph", C.c_int32), ("keep_results", C.c_int32), ("hbm_headroom_bytes", C.c_uint64)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("cancelled", C.c_uint64), ("batches", C.c_uint64), ("points", C.c_uint64),
                ("peak_out_bytes", C.c_uint64), ("spilled", C.c_uint64), ("p50_ms", C.c_double), ("p90_ms", C.c_double),
                ("p99_ms", C.c_double), ("mean_ms", C.c_double), ("max_ms", C.c_double), ("busy_s", C.c_double),
                ("worker_cpu_s", C.c_double)]


class BatchStats(C.Structure):
    _fields_ = [("records", C.c_uint64), ("seeds", C.c_uint64), ("boundary", C.c_uint64), ("points", C.c_uint64),
                ("levels", C.c_uint32)]


QUERY_NP = np.dtype([("kind", "<i4"), ("reserved", "<i4"), ("min1", "<u8"), ("max1", "<u8"), ("min2", "<u8")])

_lib = None


def lib():
    """Loads libpst_b200.so (raises PSTError if it is missing: no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not library_path.exists():
        raise PSTError(2, f"{library_path.name} is not built; run __graft_entry__.build()")
    L = C.CDLL(str(library_path))
    vp, u64, u32, i32 = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int32
    P = C.POINTER
    sigs = {
        "pst_last_error": (C.c_char_p, []),
        "pst_version": (C.c_char_p, []),
        "pst_point_size": (C.c_size_t, [i32, i32]),
        "pst_free": (i32, [vp]),
        "pst_mem_needed": (i32, [i32, i32, u64, P(u64)]),
        "pst_create": (i32, [P(vp), i32, i32, vp, u64, vp]),
        "pst_destroy": (i32, [vp]),
        "pst_image_size": (i32, [vp, P(u64)]),
        "pst_save": (i32, [vp, vp, u64, P(u64), vp]),
        "pst_load": (i32, [P(vp), vp, u64, vp]),
        "pst_save_file": (i32, [vp, C.c_char_p]),
        "pst_load_file": (i32, [P(vp), C.c_char_p, vp]),
        "pst_info": (i32, [vp, P(u64), P(u32), P(u64), P(u64), P(i32), P(i32)]),
        "pst_export": (i32, [vp, vp, vp, vp, vp, vp]),
        "pst_search": (i32, [vp, P(Query), i32, P(vp), P(u64), vp]),
        "pst_count": (i32, [vp, P(Query), P(u64), vp]),
        "pst_three_sided": (i32, [vp, u64, u64, u64, i32, P(vp), P(u64), vp]),
        "pst_two_sided_left": (i32, [vp, u64, u64, i32, P(vp), P(u64), vp]),
        "pst_two_sided_right": (i32, [vp, u64, u64, i32, P(vp), P(u64), vp]),
        "pst_search_into": (i32, [vp, P(Query), i32, vp, u64, P(u64), vp]),
        "pst_batch_create": (i32, [P(vp), vp, P(BatchOpts)]),
        "pst_batch_destroy": (i32, [vp]),
        "pst_batch_run": (i32, [vp, vp, u32, i32, i32, vp, u64, vp, P(u64), i32, vp]),
        "pst_batch_count": (i32, [vp, vp, u32, i32, vp, P(u64), vp]),
        "pst_batch_status": (i32, [vp, P(u64)]),
        "pst_batch_last_stats": (i32, [vp, P(BatchStats), vp]),
        "pst_batch_launch_shape": (i32, [vp, P(u32), P(u32), P(u32), P(u32), P(u32)]),
        "pst_ips_search": (i32, [i32, i32, vp, u64, u64, i32, P(vp), P(u64), u32, u32, vp]),
        "pst_ips_search_into": (i32, [i32, i32, vp, u64, u64, i32, vp, u64, P(u64), vp]),
        "pst_num_metacells": (i32, [P(u32), P(u32), P(u32), P(u64)]),
        "pst_server_create": (i32, [P(vp), P(ServerOpts)]),
        "pst_server_add_tree": (i32, [vp, vp, P(u32)]),
        "pst_server_add_tree_tuned": (i32, [vp, vp, P(BatchOpts), P(u32)]),
        "pst_server_submit": (i32, [vp, u32, vp, vp, i32, vp, vp]),
        "pst_server_wait": (i32, [vp, u64, u32, P(i32), P(u64)]),
        "pst_server_take": (i32, [vp, u64, vp, u64, P(u64)]),
        "pst_server_cancel": (i32, [vp, u64]),
        "pst_server_drain": (i32, [vp, u32]),
        "pst_server_get_stats": (i32, [vp, P(ServerStats)]),
        "pst_server_reset_stats": (i32, [vp]),
        "pst_server_destroy": (i32, [vp]),
        "pst_form_metacells": (i32, [i32, i32, vp, P(u32), P(u32), vp, vp]),
        "pst_read_volume": (i32, [C.c_char_p, i32, u64, vp, vp]),
        "pst_mc_tables": (i32, [vp, vp]),
        "pst_mc_count": (i32, [vp, P(u32), P(u32), vp, u64, C.c_float, P(u64), vp]),
        "pst_mc_triangles": (i32, [vp, P(u32), P(u32), vp, u64, C.c_float, vp, u64, P(u64), vp]),
        "pst_form_metacells_from_file": (i32, [C.c_char_p, i32, i32, P(u32), P(u32), vp, u64, vp]),
    }
    for name, (res, args) in sigs.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _check(st: int):
    if st != 0:
        raise PSTError(st, lib().pst_last_error().decode())


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise PSTError(2, "no CUDA device available")
    return torch


def _stream(stream=None):
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def point_dtype(dt: str, has_id: bool) -> np.dtype:
    """numpy layout of the reference's PointStruct (helpers/point-struct.h)."""
    fields = [("dim1", NP[dt]), ("dim2", NP[dt])]
    if has_id:
        fields.append(("id", np.uint32))
    return np.dtype(fields, align=True)


def value(dt: str, v) -> Value:
    x = Value()
    setattr(x, dt, NP[dt](v).item())
    return x


def value_arg(dt: str, v) -> int:
    """A pst_value passed by value.  ctypes cannot pass unions by value, but on
    x86-64 (System V) this 8-byte union of float/double/int32 is classified INTEGER
    and travels in one general-purpose register, exactly like a uint64 holding its
    bytes (4-byte members in the low half)."""
    return int.from_bytes(bytes(value(dt, v)), "little")


def points_to_device(pts: np.ndarray):
    """Copies a structured PointStruct array to a device byte tensor."""
    torch = _torch()
    raw = np.ascontiguousarray(pts).view(np.uint8).reshape(-1)
    return torch.from_numpy(raw.copy()).to("cuda")


class _DevView:
    """__cuda_array_interface__ over a raw device pointer (no ownership)."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False), "version": 3}


def _take_device_result(ptr: int, count: int, rec: np.dtype | type) -> np.ndarray:
    """Copies a library-allocated result to host memory and frees it."""
    torch = _torch()
    rec = np.dtype(rec)
    try:
        if count == 0 or not ptr:
            return np.zeros(0, rec)
        t = torch.as_tensor(_DevView(ptr, count * rec.itemsize), device="cuda")
        host = t.cpu().numpy()
        return host.view(rec).copy()
    finally:
        if ptr:
            _check(lib().pst_free(C.c_void_p(ptr)))


def free_device(ptr: int):
    """Releases a result returned by a drop-in search (pst_free)."""
    if ptr:
        _check(lib().pst_free(C.c_void_p(ptr)))


def make_queries(kinds, min1, max1, min2, dt: str) -> np.ndarray:
    """pst_query records (kind, bounds in the tree's value type)."""
    n = len(kinds)
    q = np.zeros(n, QUERY_NP)
    q["kind"] = np.asarray(kinds, np.int32)
    for f, v in (("min1", min1), ("max1", max1), ("min2", min2)):
        vals = np.asarray(v, NP[dt])
        buf = np.zeros(n, np.uint64)
        buf.view(np.uint8).reshape(n, 8)[:, :vals.itemsize] = vals.view(np.uint8).reshape(n, vals.itemsize)
        q[f] = buf
    return q


class StaticPSTGPU:
    """Mirror of the reference's StaticPSTGPU<T, PointStruct, IDType, num_IDs>
    (pst/static-pst-gpu.h:72-132).  Built from device PointStruct records."""

    def __init__(self, pts_d, num_elems: int, dt: str = "f32", has_id: bool = True, stream=None):
        self.dt, self.has_id, self.n = dt, has_id, int(num_elems)
        self._h = C.c_void_p()
        ptr = C.c_void_p(pts_d.data_ptr() if hasattr(pts_d, "data_ptr") else (pts_d or 0))
        _check(lib().pst_create(C.byref(self._h), DTYPE[dt], IDTYPE[has_id], ptr, self.n, _stream(stream)))
        self.rec_point = point_dtype(dt, has_id)

    @classmethod
    def _adopt(cls, handle: C.c_void_p):
        """Wraps a tree handle created by the library (a loaded image)."""
        self = cls.__new__(cls)
        self._h = handle
        n, lv, sl, by = C.c_uint64(), C.c_uint32(), C.c_uint64(), C.c_uint64()
        d, i = C.c_int32(), C.c_int32()
        _check(lib().pst_info(handle, C.byref(n), C.byref(lv), C.byref(sl), C.byref(by), C.byref(d), C.byref(i)))
        self.dt = {v: k for k, v in DTYPE.items()}[d.value]
        self.has_id = i.value == IDTYPE[True]
        self.n = n.value
        self.rec_point = point_dtype(self.dt, self.has_id)
        return self

    def to_bytes(self) -> bytes:
        """The tree's image (pst_save): a 64-byte header and the device arrays."""
        size = C.c_uint64()
        _check(lib().pst_image_size(self._h, C.byref(size)))
        buf = np.empty(size.value, np.uint8)
        _check(lib().pst_save(self._h, buf.ctypes.data_as(C.c_void_p), size.value, C.byref(size), _stream()))
        return buf.tobytes()

    @classmethod
    def from_bytes(cls, image: bytes):
        """Recreates a tree from its image without rebuilding it (pst_load)."""
        h = C.c_void_p()
        buf = np.frombuffer(image, np.uint8)
        _check(lib().pst_load(C.byref(h), buf.ctypes.data_as(C.c_void_p), len(buf), _stream()))
        return cls._adopt(h)

    def save(self, path):
        _check(lib().pst_save_file(self._h, str(path).encode()))

    @classmethod
    def load(cls, path):
        h = C.c_void_p()
        _check(lib().pst_load_file(C.byref(h), str(path).encode(), _stream()))
        return cls._adopt(h)

    @classmethod
    def from_numpy(cls, pts: np.ndarray, dt: str):
        has_id = "id" in pts.dtype.names
        d = points_to_device(pts)
        return cls(d, len(pts), dt, has_id)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _check(lib().pst_destroy(self._h))
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def info(self):
        n, lv, sl, by = C.c_uint64(), C.c_uint32(), C.c_uint64(), C.c_uint64()
        d, i = C.c_int32(), C.c_int32()
        _check(lib().pst_info(self._h, C.byref(n), C.byref(lv), C.byref(sl), C.byref(by), C.byref(d), C.byref(i)))
        return {"n": n.value, "levels": lv.value, "slots": sl.value, "device_bytes": by.value}

    def export(self):
        """Tree in the reference's field layout (for bit-exact comparison)."""
        S = self.info()["slots"]
        t = NP[self.dt]
        out = {"dim1": np.zeros(S, t), "dim2": np.zeros(S, t), "med": np.zeros(S, t),
               "ids": np.zeros(S, np.uint32) if self.has_id else None, "bitcodes": np.zeros(S, np.uint8)}
        p = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)  # noqa: E731
        _check(lib().pst_export(self._h, p(out["dim1"]), p(out["dim2"]), p(out["med"]), p(out["ids"]),
                                p(out["bitcodes"])))
        return out

    def _ret(self, ret):
        r = ret if isinstance(ret, str) else ("ids" if ret is np.uint32 else "points")
        return r, (np.uint32 if r == "ids" else self.rec_point)

    def count(self, kind: str, min1=0, max1=0, min2=0, stream=None) -> int:
        """Number of points the query reports (pst_count), without producing them."""
        q = Query(KIND[kind], 0, value(self.dt, min1), value(self.dt, max1), value(self.dt, min2))
        cnt = C.c_uint64()
        _check(lib().pst_count(self._h, C.byref(q), C.byref(cnt), _stream(stream)))
        return cnt.value

    def search_device(self, kind: str, min1=0, max1=0, min2=0, ret="ids", stream=None):
        """The drop-in call itself: returns (device pointer, count) of the
        library-allocated result, which the caller releases with free_device (the
        reference's searches hand back a cudaMalloc'd array the same way)."""
        r, _ = self._ret(ret)
        q = Query(KIND[kind], 0, value(self.dt, min1), value(self.dt, max1), value(self.dt, min2))
        out, cnt = C.c_void_p(), C.c_uint64()
        _check(lib().pst_search(self._h, C.byref(q), RET[r], C.byref(out), C.byref(cnt), _stream(stream)))
        return out.value or 0, cnt.value

    def search(self, kind: str, min1=0, max1=0, min2=0, ret="ids", stream=None) -> np.ndarray:
        """One query through the drop-in call (callee-allocated result)."""
        r, rec = self._ret(ret)
        q = Query(KIND[kind], 0, value(self.dt, min1), value(self.dt, max1), value(self.dt, min2))
        out, cnt = C.c_void_p(), C.c_uint64()
        _check(lib().pst_search(self._h, C.byref(q), RET[r], C.byref(out), C.byref(cnt), _stream(stream)))
        return _take_device_result(out.value or 0, cnt.value, rec)

    # reference names (pst/static-pst-gpu.h:103-128)
    def threeSidedSearch(self, min_dim1_val, max_dim1_val, min_dim2_val, ret="points"):
        r, rec = self._ret(ret)
        out, cnt = C.c_void_p(), C.c_uint64()
        _check(lib().pst_three_sided(self._h, value_arg(self.dt, min_dim1_val), value_arg(self.dt, max_dim1_val),
                                     value_arg(self.dt, min_dim2_val), RET[r], C.byref(out), C.byref(cnt), _stream()))
        return _take_device_result(out.value or 0, cnt.value, rec)

    def twoSidedLeftSearch(self, max_dim1_val, min_dim2_val, ret="points"):
        r, rec = self._ret(ret)
        out, cnt = C.c_void_p(), C.c_uint64()
        _check(lib().pst_two_sided_left(self._h, value_arg(self.dt, max_dim1_val), value_arg(self.dt, min_dim2_val),
                                        RET[r], C.byref(out), C.byref(cnt), _stream()))
        return _take_device_result(out.value or 0, cnt.value, rec)

    def twoSidedRightSearch(self, min_dim1_val, min_dim2_val, ret="points"):
        r, rec = self._ret(ret)
        out, cnt = C.c_void_p(), C.c_uint64()
        _check(lib().pst_two_sided_right(self._h, value_arg(self.dt, min_dim1_val), value_arg(self.dt, min_dim2_val),
                                         RET[r], C.byref(out), C.byref(cnt), _stream()))
        return _take_device_result(out.value or 0, cnt.value, rec)

    def search_into(self, kind: str, out_d, capacity: int, min1=0, max1=0, min2=0, ret="ids", stream=None) -> int:
        r, _ = self._ret(ret)
        q = Query(KIND[kind], 0, value(self.dt, min1), value(self.dt, max1), value(self.dt, min2))
        cnt = C.c_uint64()
        st = lib().pst_search_into(self._h, C.byref(q), RET[r], C.c_void_p(out_d.data_ptr()), capacity,
                                   C.byref(cnt), _stream(stream))
        if st == 4:
            return -int(cnt.value)
        _check(st)
        return int(cnt.value)

    @staticmethod
    def calcGlobalMemNeeded(num_elems: int, dt: str = "f32", has_id: bool = True) -> int:
        b = C.c_uint64()
        _check(lib().pst_mem_needed(DTYPE[dt], IDTYPE[has_id], num_elems, C.byref(b)))
        return b.value


class StaticPSTGPUArr(StaticPSTGPU):
    """Mirror of StaticPSTGPUArr (pst/static-pst-gpu-arr.h:45-103).  The reference
    splits the input into per-block shallow trees and implements only
    twoSidedLeftSearch; here the same surface runs on the one complete tree, so its
    3-sided and 2-sided-right searches work too and every result equals the
    reference's StaticPSTCPUIter."""

    def __init__(self, pts_d, num_elems: int, threads_per_block: int = 128, dt: str = "f32", has_id: bool = True,
                 stream=None):
        super().__init__(pts_d, num_elems, dt, has_id, stream)
        self.threads_per_block = threads_per_block


class BatchEngine:
    """Batched queries on one resident tree (pst_batch_*).

    The launch shape (block_threads, blocks_per_sm, emit_records,
    top_pass_queries; 0 = the library's default) comes from the arguments, or from
    `tuning`: a dict of those fields (what autotune.tune returns), or "cache" for the
    autotuner's cached choice for this tree shape and batch size (the defaults when
    it has none)."""

    def __init__(self, tree: StaticPSTGPU, max_queries: int, task_capacity: int = 0, use_graph: bool = True,
                 blocks_per_sm: int = 0, block_threads: int = 0, emit_records: int = 0, top_pass_queries: int = 0,
                 tuning=None):
        self.tree = tree
        self.max_queries = max_queries
        shape = {"block_threads": block_threads, "blocks_per_sm": blocks_per_sm, "emit_records": emit_records,
                 "top_pass_queries": top_pass_queries}
        if tuning == "cache":
            from .autotune import cached
            tuning = cached(tree, max_queries)
        if tuning:
            shape.update({k: int(tuning[k]) for k in TUNING_FIELDS if k in tuning})
            use_graph = bool(tuning.get("use_graph", use_graph))
        self.shape = dict(shape, use_graph=bool(use_graph))
        o = BatchOpts(max_queries, task_capacity, shape["block_threads"], shape["blocks_per_sm"], int(use_graph),
                      shape["emit_records"], shape["top_pass_queries"])
        self._h = C.c_void_p()
        _check(lib().pst_batch_create(C.byref(self._h), tree.handle, C.byref(o)))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _check(lib().pst_batch_destroy(self._h))
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def launch_shape(self) -> dict:
        """The engine's launch shape as resolved on the device (pst_batch_launch_shape)."""
        t, b, g, e, q = (C.c_uint32() for _ in range(5))
        _check(lib().pst_batch_launch_shape(self._h, C.byref(t), C.byref(b), C.byref(g), C.byref(e), C.byref(q)))
        return {"block_threads": t.value, "blocks_per_sm": b.value, "grid": g.value, "emit_records": e.value,
                "top_pass_queries": q.value}

    def last_stats(self) -> dict:
        st = BatchStats()
        per = (C.c_uint32 * 40)()
        _check(lib().pst_batch_last_stats(self._h, C.byref(st), per))
        d = {f: getattr(st, f) for f, _ in BatchStats._fields_}
        d["per_level"] = list(per)[: st.levels]
        return d

    def count(self, queries: np.ndarray, stream=None):
        torch = _torch()
        nq = len(queries)
        counts = torch.zeros(max(nq, 1), dtype=torch.int64, device="cuda")
        tot = C.c_uint64()
        q = np.ascontiguousarray(queries)
        _check(lib().pst_batch_count(self._h, q.ctypes.data_as(C.c_void_p), nq, 0, C.c_void_p(counts.data_ptr()),
                                     C.byref(tot), _stream(stream)))
        return counts[:nq], tot.value

    def run(self, queries, out_d, offsets_d, ret="ids", queries_on_device=False, sync=True, stream=None):
        """Returns (status, total).  queries: host numpy pst_query array or device tensor."""
        if queries_on_device:
            nq = queries.numel() * queries.element_size() // QUERY_NP.itemsize
            qp = C.c_void_p(queries.data_ptr())
        else:
            queries = np.ascontiguousarray(queries)
            nq = len(queries)
            qp = queries.ctypes.data_as(C.c_void_p)
        rec = 4 if ret == "ids" else self.tree.rec_point.itemsize
        cap = out_d.numel() * out_d.element_size() // rec
        tot = C.c_uint64()
        st = lib().pst_batch_run(self._h, qp, nq, int(queries_on_device), RET[ret], C.c_void_p(out_d.data_ptr()),
                                 cap, C.c_void_p(offsets_d.data_ptr()), C.byref(tot), int(sync), _stream(stream))
        if st not in (0, 4):
            _check(st)
        return st, tot.value

    def search(self, queries: np.ndarray, ret="ids"):
        """Convenience: returns (offsets, results) on the host."""
        torch = _torch()
        counts, total = self.count(queries)
        rec = np.uint32 if ret == "ids" else self.tree.rec_point
        rsz = np.dtype(rec).itemsize
        out = torch.empty(max(total * rsz, 16), dtype=torch.uint8, device="cuda")
        offs = torch.empty(len(queries) + 1, dtype=torch.int64, device="cuda")
        st, tot = self.run(queries, out, offs, ret=ret)
        _check(st)
        torch.cuda.synchronize()
        res = out[: tot * rsz].cpu().numpy().view(rec)
        return offs.cpu().numpy().astype(np.uint64), res


class Server:
    """Serving loop over resident trees (pst_server_*)."""

    def __init__(self, max_batch=1024, slots_per_tree=2, out_budget_bytes=1 << 30, use_graph=True,
                 keep_results=1, hbm_headroom_bytes=0):
        keep_results = int(keep_results)
        self.keep_results = keep_results
        self.max_batch = max_batch or 1024
        o = ServerOpts(max_batch, slots_per_tree, out_budget_bytes, int(use_graph), int(keep_results),
                       int(hbm_headroom_bytes))
        self._h = C.c_void_p()
        _check(lib().pst_server_create(C.byref(self._h), C.byref(o)))
        self.trees = []

    def add_tree(self, tree: StaticPSTGPU, tuning=None) -> int:
        """Registers a resident tree; `tuning` sets its engines' launch shape (a dict
        of BatchOpts launch fields, or "cache" for the autotuner's cached choice)."""
        idx = C.c_uint32()
        if tuning == "cache":
            from .autotune import cached
            tuning = cached(tree, self.max_batch)
        if tuning:
            o = BatchOpts(0, 0, *(int(tuning.get(k, 0)) for k in ("block_threads", "blocks_per_sm")), 0,
                          int(tuning.get("emit_records", 0)), int(tuning.get("top_pass_queries", 0)))
            _check(lib().pst_server_add_tree_tuned(self._h, tree.handle, C.byref(o), C.byref(idx)))
        else:
            _check(lib().pst_server_add_tree(self._h, tree.handle, C.byref(idx)))
        self.trees.append(tree)
        return idx.value

    def submit(self, tree_index, queries: np.ndarray, ret="ids", arrival_ns=None) -> np.ndarray:
        """Queues requests; tree_index is an int or an array (one per query)."""
        q = np.ascontiguousarray(queries)
        n = len(q)
        ti = np.ascontiguousarray(np.broadcast_to(np.asarray(tree_index, np.uint32), (n,)))
        ids = np.zeros(n, np.uint64)
        arr = None if arrival_ns is None else np.ascontiguousarray(np.asarray(arrival_ns, np.uint64))
        p = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)  # noqa: E731
        _check(lib().pst_server_submit(self._h, n, p(ti), p(q), RET[ret], p(arr), p(ids)))
        return ids

    def wait(self, rid: int, timeout_ms: int = 10000):
        """Returns (status, count) or raises PSTError(PST_ERR_TIMEOUT)."""
        st, cnt = C.c_int32(), C.c_uint64()
        _check(lib().pst_server_wait(self._h, int(rid), timeout_ms, C.byref(st), C.byref(cnt)))
        return st.value, cnt.value

    def take(self, rid: int, rec) -> np.ndarray:
        _, cnt = self.wait(rid)
        rec = np.dtype(rec)
        out = np.zeros(max(cnt, 1), rec)
        c = C.c_uint64()
        _check(lib().pst_server_take(self._h, int(rid), out.ctypes.data_as(C.c_void_p) if self.keep_results == 1 else None,
                                     len(out), C.byref(c)))
        return out[: c.value]

    def cancel(self, rid: int):
        _check(lib().pst_server_cancel(self._h, int(rid)))

    def drain(self, timeout_ms: int = 60000):
        _check(lib().pst_server_drain(self._h, timeout_ms))

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().pst_server_get_stats(self._h, C.byref(st)))
        return {f: getattr(st, f) for f, _ in ServerStats._fields_}

    def reset_stats(self):
        _check(lib().pst_server_reset_stats(self._h))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _check(lib().pst_server_destroy(self._h))
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def intervalParallelSearch(pts_d, num_elems: int, search_val, dt: str = "f32", has_id: bool = True, ret="ids",
                           num_thread_blocks: int = 0, threads_per_block: int = 0, stream=None) -> np.ndarray:
    """Mirror of intervalParallelSearch (interval-parallel-search/interval-parallel-search.h:29)."""
    out, cnt = C.c_void_p(), C.c_uint64()
    _check(lib().pst_ips_search(DTYPE[dt], IDTYPE[has_id], C.c_void_p(pts_d.data_ptr()), num_elems,
                                value_arg(dt, search_val), RET[ret], C.byref(out), C.byref(cnt), num_thread_blocks,
                                threads_per_block, _stream(stream)))
    rec = np.uint32 if ret == "ids" else point_dtype(dt, has_id)
    return _take_device_result(out.value or 0, cnt.value, rec)


def calcNumMetacells(pt_grid_dims, metacell_dims):
    """Mirror of calcNumMetacells (helpers/isosurface-data-processing.h:23-36)."""
    P = (C.c_uint32 * 3)(*pt_grid_dims)
    M = (C.c_uint32 * 3)(*metacell_dims)
    G = (C.c_uint32 * 3)()
    n = C.c_uint64()
    _check(lib().pst_num_metacells(P, M, G, C.byref(n)))
    return list(G), n.value


def formMetacellTags(vert_d, pt_grid_dims, metacell_dims, dt: str = "f32", has_id: bool = True, stream=None):
    """Mirror of formMetacellTags (helpers/isosurface-data-processing.h:69-137): returns a
    device byte tensor of PointStruct records, one per metacell, indexed by metacell id."""
    torch = _torch()
    _, n = calcNumMetacells(pt_grid_dims, metacell_dims)
    rec = point_dtype(dt, has_id)
    out = torch.empty(max(n * rec.itemsize, 16), dtype=torch.uint8, device="cuda")
    P = (C.c_uint32 * 3)(*pt_grid_dims)
    M = (C.c_uint32 * 3)(*metacell_dims)
    _check(lib().pst_form_metacells(DTYPE[dt], IDTYPE[has_id], C.c_void_p(vert_d.data_ptr()), P, M,
                                    C.c_void_p(out.data_ptr()), _stream(stream)))
    return out[: n * rec.itemsize], n


def readInVertices(path, num_vertices: int, dt: str = "f32", stream=None):
    """Mirror of readInVertices (helpers/isosurface-data-processing.h:205-229), reading
    the raw volume straight into a device tensor (pst_read_volume)."""
    torch = _torch()
    tt = {"f32": torch.float32, "f64": torch.float64, "i32": torch.int32}[dt]
    out = torch.empty(max(int(num_vertices), 1), dtype=tt, device="cuda")
    _check(lib().pst_read_volume(str(path).encode(), DTYPE[dt], int(num_vertices), C.c_void_p(out.data_ptr()),
                                 _stream(stream)))
    return out[: int(num_vertices)]


def formMetacellTagsFromFile(path, pt_grid_dims, metacell_dims, dt: str = "f32", has_id: bool = True,
                             slab_bytes: int = 0, stream=None):
    """readInVertices + formMetacellTags in one stream (pst_form_metacells_from_file):
    the volume never sits on the device whole; returns (records, n) like
    formMetacellTags."""
    torch = _torch()
    _, n = calcNumMetacells(pt_grid_dims, metacell_dims)
    rec = point_dtype(dt, has_id)
    out = torch.empty(max(n * rec.itemsize, 16), dtype=torch.uint8, device="cuda")
    P = (C.c_uint32 * 3)(*pt_grid_dims)
    M = (C.c_uint32 * 3)(*metacell_dims)
    _check(lib().pst_form_metacells_from_file(str(path).encode(), DTYPE[dt], IDTYPE[has_id], P, M,
                                              C.c_void_p(out.data_ptr()), int(slab_bytes), _stream(stream)))
    return out[: n * rec.itemsize], n


def marchingCubesTables():
    """The library's triangle table: (ntri[256], edges[256, 15]) uint8."""
    ntri = np.zeros(256, np.uint8)
    edges = np.zeros((256, 15), np.uint8)
    _check(lib().pst_mc_tables(ntri.ctypes.data_as(C.c_void_p), edges.ctypes.data_as(C.c_void_p)))
    return ntri, edges


def marchingCubes(vol_d, pt_grid_dims, metacell_dims, ids_d, iso: float, stream=None):
    """Triangles (n, 9) float32 on the device of the cells of the metacells ids_d
    (a device uint32 tensor, e.g. a twoSidedLeftSearch(iso, iso) result)."""
    torch = _torch()
    P = (C.c_uint32 * 3)(*pt_grid_dims)
    M = (C.c_uint32 * 3)(*metacell_dims)
    n_ids = int(ids_d.numel()) if ids_d is not None else 0
    vp = C.c_void_p(vol_d.data_ptr())
    ip = C.c_void_p(ids_d.data_ptr() if n_ids else 0)
    cnt = C.c_uint64()
    _check(lib().pst_mc_count(vp, P, M, ip, n_ids, float(iso), C.byref(cnt), _stream(stream)))
    out = torch.empty((max(cnt.value, 1), 9), dtype=torch.float32, device="cuda")
    got = C.c_uint64()
    _check(lib().pst_mc_triangles(vp, P, M, ip, n_ids, float(iso), C.c_void_p(out.data_ptr()), cnt.value,
                                  C.byref(got), _stream(stream)))
    return out[: got.value]


def _env_flag(name: str) -> bool:
    return os.environ.get(name, "") not in ("", "0")
