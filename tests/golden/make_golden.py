"""Generates tests/golden/reference_trees.npz from the reference itself:
StaticPSTCPUIter compiled unmodified from its sources (oracle/_ref/libpstref.so,
built by `make -C oracle`).  For each seeded case it stores the input points, the
reference's whole tree (its field layout) and the results of a few queries.

  python tests/golden/make_golden.py
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent / "oracle"))
sys.path.insert(0, str(HERE.parent))

import oracle  # noqa: E402
from datagen import rand_points, rand_queries  # noqa: E402

CASES = [(dt, ids, n, dup) for dt in ("f32", "f64", "i32") for ids in ("arange", "random", "none")
         for n, dup in ((0, False), (1, False), (2, True), (5, True), (33, True), (100, False), (1000, True))]


def main():
    if not oracle.Ref.available():
        raise SystemExit("build oracle/_ref first: make -C oracle")
    out = {}
    for ci, (dt, ids, n, dup) in enumerate(CASES):
        pts = rand_points(n, dt, ids=ids, dup=dup, seed=500 + ci)
        ref = oracle.Ref(pts, dt)
        tr = ref.export()
        key = f"c{ci}"
        out[f"{key}_meta"] = np.array([ci, n, ("f32", "f64", "i32").index(dt), int(ids != "none")], np.int64)
        out[f"{key}_points"] = pts.view(np.uint8).reshape(-1)
        for f in ("dim1", "dim2", "med", "bitcodes"):
            out[f"{key}_{f}"] = getattr(tr, f)
        if tr.has_id:
            out[f"{key}_ids"] = tr.ids
        qs = rand_queries(pts, 6, seed=ci)
        qarr = np.zeros((len(qs), 4), np.float64)
        for qi, (kind, a, b, m2) in enumerate(qs):
            qarr[qi] = [oracle.KINDS[kind], a, b, m2]
            res = ref.search(kind, a, b, m2, points=True)
            out[f"{key}_q{qi}"] = oracle.canon(res)
        out[f"{key}_queries"] = qarr
        ref.close()
    np.savez_compressed(HERE / "reference_trees.npz", **out)
    print(f"wrote {len(CASES)} cases")


if __name__ == "__main__":
    main()
