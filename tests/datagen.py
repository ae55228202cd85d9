"""Seeded synthetic inputs shared by the tests (numpy Generator, PCG64)."""
from __future__ import annotations

import numpy as np

from oracle import make_points


def rand_points(n: int, dt: str = "f32", ids: str = "arange", dup: bool = False, seed: int = 1,
                lo: float = 0.0, hi: float = 1000.0, width: float = 50.0, signed_zero: bool = False):
    """dim1 ~ U[lo, hi), dim2 = dim1 + U[0, width) in the value type.

    ids: "arange" (0..n-1), "random" (with duplicates), "desc" (n-1..0, so not
    non-decreasing), "const" (all equal) or "none" (id-less records).
    dup: draw from a small value set so that ties are everywhere."""
    rng = np.random.default_rng(seed)
    if dt == "i32":
        if dup:
            d1 = rng.integers(-20, 20, n).astype(np.int32)
            d2 = (d1 + rng.integers(0, 8, n)).astype(np.int32)
        else:
            d1 = rng.integers(int(lo), int(hi) if hi > lo + 1 else int(lo) + 2, n).astype(np.int32)
            d2 = (d1 + rng.integers(0, max(int(width), 1), n)).astype(np.int32)
    else:
        t = np.float32 if dt == "f32" else np.float64
        if dup:
            d1 = rng.integers(-20, 20, n).astype(t) * t(0.5)
            d2 = d1 + rng.integers(0, 8, n).astype(t) * t(0.5)
        else:
            d1 = (rng.random(n) * (hi - lo) + lo).astype(t)
            d2 = (d1 + (rng.random(n) * width).astype(t)).astype(t)
        if signed_zero and n:
            z = rng.random(n) < 0.2
            d1[z] = t(-0.0) if rng.random() < 0.5 else t(0.0)
            d1[z & (rng.random(n) < 0.5)] = t(-0.0)
            d2[z] = np.where(rng.random(int(z.sum())) < 0.5, t(-0.0), t(0.0))
    if ids == "none":
        idv = None
    elif ids == "arange":
        idv = np.arange(n, dtype=np.uint32)
    elif ids == "desc":
        idv = np.arange(n, dtype=np.uint32)[::-1].copy()
    elif ids == "const":
        idv = np.full(n, 7, np.uint32)
    else:
        idv = rng.integers(0, max(n // 3, 1), n).astype(np.uint32)
    return make_points(d1, d2, idv, dt)


def rand_queries(pts: np.ndarray, k: int, seed: int = 2):
    """k queries of mixed kinds with bounds drawn from the data's own values."""
    rng = np.random.default_rng(seed)
    d1, d2 = pts["dim1"], pts["dim2"]
    out = []
    if len(pts) == 0:
        return [("three", 0, 0, 0)] * k
    for _ in range(k):
        kind = ["three", "left", "right"][rng.integers(0, 3)]
        a, b = sorted(rng.choice(d1, 2))
        m2 = rng.choice(d2)
        if rng.random() < 0.1:
            m2 = rng.choice(d1)
        out.append((kind, a, b, m2))
    return out


def blob_volume(px: int, py: int, pz: int, nblobs: int = 32, seed: int = 1, noise: float = 0.01,
                sigma=(8.0, 40.0), amp=(0.5, 1.0)) -> np.ndarray:
    """Sum of isotropic Gaussian blobs (centres uniform over the grid, sigma and
    amplitude uniform in the given ranges) plus N(0, noise) in float32, shape
    (pz, py, px), x fastest.  Each blob is evaluated separably over its 4-sigma box."""
    rng = np.random.default_rng(seed)
    vol = np.zeros((pz, py, px), np.float32)
    for _ in range(nblobs):
        c = rng.uniform([0, 0, 0], [px, py, pz])
        s = rng.uniform(*sigma)
        a = np.float32(rng.uniform(*amp))
        lo = np.maximum(np.floor(c - 4 * s).astype(int), 0)
        hi = np.minimum(np.ceil(c + 4 * s).astype(int) + 1, [px, py, pz])
        g = [np.exp(-0.5 * ((np.arange(lo[i], hi[i]) - c[i]) / s) ** 2).astype(np.float32) for i in range(3)]
        vol[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] += a * (g[2][:, None, None] * g[1][None, :, None] * g[0][None, None, :])
    vol += rng.normal(0.0, noise, vol.shape).astype(np.float32)
    return vol
