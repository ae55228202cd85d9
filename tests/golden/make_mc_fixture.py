"""Generates tests/golden/mc_reference_cases.npz from the reference's isosurface
sample (.marching-cubes/marchingCubes_kernel.cu and .marching-cubes/tables.h,
NVIDIA's marching-cubes sample shipped inside the reference), by reading those
files as text.  Run it where the reference checkout is present:

    python tests/golden/make_mc_fixture.py [path to the reference checkout]

It stores what the sample's tables say about each of the 256 cube cases, not the
tables themselves:
  * corners: the sample's corner offsets v[0..7] (marchingCubes_kernel.cu:283-290),
  * edge_corners: the two corners of each of its 12 edges (the vertexInterp calls,
    marchingCubes_kernel.cu:354-367),
  * below_bit: cube index bit i is set when corner i is below the isovalue
    (marchingCubes_kernel.cu:309-317),
  * tri_edge_mask[c]: the 12-bit set of edges that triTable[c] places vertices on,
  * edge_table[c]: edgeTable[c] (the sample's own crossed-edge mask),
  * num_verts[c]: numVertsTable[c] (three per triangle).
"""
from __future__ import annotations

import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _ints(block: str) -> list[int]:
    vals = []
    for tok in re.findall(r"0x[0-9a-fA-F]+|-?\d+|\bX\b", block):
        vals.append(-1 if tok == "X" else int(tok, 0))
    return vals


def _array(text: str, name: str) -> list[int]:
    m = re.search(name + r"\s*(\[\d+\])+\s*=\s*\{", text)
    if not m:
        raise SystemExit(f"{name} not found")
    depth, i = 0, m.end() - 1
    for j in range(i, len(text)):
        depth += text[j] == "{"
        depth -= text[j] == "}"
        if depth == 0:
            return _ints(text[i:j + 1])
    raise SystemExit(f"{name} not terminated")


def main(ref_root: Path):
    mcdir = ref_root / ".marching-cubes"
    tables = (mcdir / "tables.h").read_text()
    kernel = (mcdir / "marchingCubes_kernel.cu").read_text()
    # drop comments so that only the initialisers are read
    tables = re.sub(r"//[^\n]*|/\*.*?\*/", "", tables, flags=re.S)
    tri = np.array(_array(tables, "triTable"), np.int64).reshape(256, 16)
    edge_table = np.array(_array(tables, "edgeTable"), np.int64)
    num_verts = np.array(_array(tables, "numVertsTable"), np.int64)
    assert edge_table.shape == (256,) and num_verts.shape == (256,)

    corners = np.zeros((8, 3), np.int64)
    for i, body in re.findall(r"v\[(\d)\]\s*=\s*p\s*\+\s*make_float3\(([^)]*)\)", kernel):
        corners[int(i)] = [0 if t.strip() == "0" else 1 for t in body.split(",")]
    pairs = {}
    for e, a, b in re.findall(r"vertlist\[(\d+)\]\s*=\s*vertexInterp\(\s*isoValue,\s*v\[(\d)\],\s*v\[(\d)\]", kernel):
        pairs[int(e)] = (int(a), int(b))
    assert sorted(pairs) == list(range(12)), pairs
    edge_corners = np.array([pairs[e] for e in range(12)], np.int64)
    below = re.findall(r"cubeindex\s*\+?=\s*uint\(field\[(\d)\]\s*<\s*isoValue\)(?:\s*\*\s*(\d+))?", kernel)
    below_bit = np.zeros(8, np.int64)
    for c, mul in below[:8]:
        below_bit[int(c)] = (int(mul) if mul else 1).bit_length() - 1

    mask = np.zeros(256, np.int64)
    for c in range(256):
        for e in tri[c]:
            if e >= 0 and e != 255:
                mask[c] |= 1 << int(e)
    np.savez_compressed(HERE / "mc_reference_cases.npz", corners=corners, edge_corners=edge_corners,
                        below_bit=below_bit, tri_edge_mask=mask.astype(np.uint16),
                        edge_table=edge_table.astype(np.uint16), num_verts=num_verts.astype(np.uint8))
    print("wrote", HERE / "mc_reference_cases.npz")


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else HERE.parents[2] / "reference")
