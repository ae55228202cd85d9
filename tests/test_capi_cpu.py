"""CPU checks of the C ABI library: it loads without a GPU, exports every symbol
include/pst_c.h declares, and its no-device paths fail loudly (no fallback)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    text = (ROOT / "include" / "pst_c.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pst_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ["pst_create", "pst_destroy", "pst_search", "pst_three_sided", "pst_two_sided_left",
                 "pst_two_sided_right", "pst_batch_run", "pst_ips_search", "pst_form_metacells",
                 "pst_num_metacells", "pst_mem_needed", "pst_export"]:
        assert must in names


def test_library_exports_every_declared_symbol(pst):
    lib = pst.lib()
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_point_sizes_match_reference_layout(pst, oracle):
    lib = pst.lib()
    for dt, code in (("f32", 0), ("f64", 1), ("i32", 2)):
        for has_id in (False, True):
            assert lib.pst_point_size(code, int(has_id)) == oracle.point_dtype(dt, has_id).itemsize
    assert lib.pst_point_size(7, 0) == 0


def test_host_only_entry_points(pst):
    """calcNumMetacells and memory sizing need no device."""
    grid, n = pst.calcNumMetacells([512, 512, 512], [4, 4, 4])
    assert grid == [128, 128, 128] and n == 128 ** 3
    grid, n = pst.calcNumMetacells([600, 248, 248], [4, 4, 4])
    assert grid == [150, 62, 62]
    lib = pst.lib()
    b = C.c_uint64()
    assert lib.pst_mem_needed(0, 1, 1 << 20, C.byref(b)) == 0 and b.value > (1 << 20) * 17
    assert lib.pst_mem_needed(9, 1, 10, C.byref(b)) == 1


def test_no_device_fails_loudly(pst):
    import torch
    if torch.cuda.is_available():
        return
    lib = pst.lib()
    h = C.c_void_p()
    st = lib.pst_create(C.byref(h), 0, 1, None, 10, None)
    assert st == 2 and b"CUDA" in lib.pst_last_error()


def test_query_record_layout(pst):
    q = pst.make_queries([0, 1], [1.5, 2.0], [3.0, 4.0], [-1.0, 7.0], "f32")
    assert q.dtype.itemsize == C.sizeof(pst.pst.Query) == 32
    raw = q.view(np.uint8).reshape(2, 32)
    assert np.frombuffer(raw[0, 8:12].tobytes(), np.float32)[0] == 1.5
    q64 = pst.make_queries([2], [0.1], [0.2], [0.3], "f64")
    assert np.frombuffer(q64.view(np.uint8)[8:16].tobytes(), np.float64)[0] == 0.1
