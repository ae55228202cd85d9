"""The oracle against golden vectors produced by the reference itself
(tests/golden/make_golden.py): whole trees and query results, bit for bit."""
from pathlib import Path

import numpy as np
import pytest

import oracle

GOLDEN = Path(__file__).resolve().parent / "golden" / "reference_trees.npz"
DTS = ("f32", "f64", "i32")
KIND_NAMES = {v: k for k, v in oracle.KINDS.items()}


def cases():
    z = np.load(GOLDEN)
    ids = sorted({k.split("_")[0] for k in z.files}, key=lambda s: int(s[1:]))
    return z, ids


def load_case(z, key):
    ci, n, dti, has_id = z[f"{key}_meta"]
    dt = DTS[dti]
    pts = z[f"{key}_points"].view(oracle.point_dtype(dt, bool(has_id)))
    return dt, bool(has_id), pts


def test_golden_trees_and_queries():
    z, keys = cases()
    assert len(keys) >= 60
    for key in keys:
        dt, has_id, pts = load_case(z, key)
        mine = oracle.Orc.build(pts, dt)
        for f in ("dim1", "dim2", "med", "bitcodes"):
            assert getattr(mine, f).tobytes() == z[f"{key}_{f}"].tobytes(), (key, f)
        if has_id:
            assert mine.ids.tobytes() == z[f"{key}_ids"].tobytes(), key
        for qi, (kind, a, b, m2) in enumerate(z[f"{key}_queries"]):
            t = oracle.DTYPES[dt]
            got = oracle.canon(oracle.Orc.search_points(mine, KIND_NAMES[int(kind)], t(a), t(b), t(m2)))
            assert np.array_equal(got, z[f"{key}_q{qi}"]), (key, qi)


@pytest.mark.gpu
def test_golden_gpu_trees(pst):
    """The GPU tree equals the reference's own tree on every golden case."""
    z, keys = cases()
    for key in keys:
        dt, has_id, pts = load_case(z, key)
        if len(pts) == 0:
            continue
        ex = pst.StaticPSTGPU.from_numpy(pts.copy(), dt).export()
        for f in ("dim1", "dim2", "med", "bitcodes"):
            assert ex[f].tobytes() == z[f"{key}_{f}"].tobytes(), (key, f)
        if has_id:
            assert ex["ids"].tobytes() == z[f"{key}_ids"].tobytes(), key
