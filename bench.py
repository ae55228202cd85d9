"""Benchmark of the static priority search tree hot path on B200.

Workload (one "step" = one batched launch): 4096 queries (50% 3-sided, 25% 2-sided
left, 25% 2-sided right) with target selectivities log-uniform in [1e-7, 1e-2], on
a resident tree of 2^28 float32 points with uint32 ids, dim1 ~ U[0, 2^24) and
dim2 = dim1 + U[0, 2^16) (seeded synthetic data; the tree alone is 7.1 GiB, far
larger than L2, so no flush is needed between steps).  Query bounds are fixed
once by bisection on exact counts.

Metric: points reported per second (value: inputs resident in HBM, results to a
device buffer; e2e: the same call from host memory with the query upload and the
result download inside the timed region).  The engine's launch shape is picked by
the project's autotuner on the step's queries before timing.

Beside the headline, the line carries: the same tree under 4096 queries over
disjoint ranges (every point reported once), the 2^26 exponential-gap
configuration against 4096 plain launches, construction with its roofline, the
2^28 large-random-tree matrix and interval scans, the 512^3 isosurface pipeline,
serving over 8 resident trees, and the reference's CPU search timed on a sample.

With N > 1 ranks (torchrun) each rank holds one dim1 shard of one point set
(weak scaling) and answers the queries routed to it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import ctypes as C

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG_DIR = ROOT / "static-priority-search-tree_b200"
sys.path.insert(0, str(ROOT / "oracle"))

METRIC = "reported pts/s & queries/s at 2^28 pts, batched vs per-query; serving p50/p99 ms"
UNIT = "pts/s"
N_POINTS = 1 << 28
NQ = 4096
SEL_LO, SEL_HI = 1e-7, 1e-2
# Algorithmic bytes per reported point, float32 tree returning ids: dim1 and dim2
# read (4 + 4), id read (4), id written (4).  A point inside a report-above subtree
# needs no dim1 test, so the search can move as little as 12 B per point.
BYTES_PER_PT = 16
BYTES_PER_PT_MIN = 12


_T0 = time.perf_counter()


def log(msg):
    """Progress on stderr (stdout carries only the JSON line)."""
    print(f"[bench {time.perf_counter() - _T0:7.1f}s] {msg}", file=sys.stderr, flush=True)


def load_package():
    if "pst_b200" in sys.modules:
        return sys.modules["pst_b200"]
    spec = importlib.util.spec_from_file_location("pst_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["pst_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# data

def gen_points_device(n, seed, torch):
    """(n, 3) int32 tensor = PointStruct<float, uint32_t, 1> records."""
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    d1 = torch.rand(n, generator=g, device="cuda", dtype=torch.float32) * float(1 << 24)
    d2 = d1 + torch.rand(n, generator=g, device="cuda", dtype=torch.float32) * float(1 << 16)
    rec = torch.empty((n, 3), dtype=torch.int32, device="cuda")
    rec[:, 0] = d1.view(torch.int32)
    rec[:, 1] = d2.view(torch.int32)
    rec[:, 2] = torch.arange(n, device="cuda", dtype=torch.int32)
    del d1, d2
    return rec


SLAB = float(1 << 24)  # dim1 width of one shard's slab


def slab_points_device(n, rank, torch):
    """Shard `rank` of the sharded point set (weak scaling: every shard holds 2^28
    points): the large-random-tree distribution with dim1 ~ U[r 2^24, (r + 1) 2^24)
    (float32, shifted after drawing), dim2 = dim1 + U[0, 2^16), ids r n ..
    (r + 1) n - 1.  Shard 0 is the one-GPU workload itself."""
    rec = gen_points_device(n, seed=1 + rank, torch=torch)
    if rank:
        vals = rec[:, :2].view(torch.float32)
        vals += float(rank) * SLAB
        rec[:, 2] += rank * n
    return rec


def slab_bounds(rec, torch):
    """(min dim1, max dim1, max dim2, nonempty) of a (n, 3) float32-with-id slab."""
    v = rec[:, :2].view(torch.float32)
    return (float(v[:, 0].min().item()), float(v[:, 0].max().item()), float(v[:, 1].max().item()), 1.0)


def sharded_block(count_fn, rank, world, n, seed_base=7):
    """This shard's block of the global query list: the mixed plan of the one-GPU
    workload inside the shard's slab, bisected on the shard's own counts.  A
    2-sided-right query of small selectivity reports a suffix of the dim1 order, so
    only the last shard keeps its right queries as they are; on every other shard
    they become 3-sided queries clipped at the slab's top (the same points the right
    query finds on that shard's slab).  Returns (kinds, min1, max1, min2, sel)."""
    kinds, sel, anchor = query_plan(NQ, seed_base + rank)
    origin = float(rank) * SLAB
    min1, max1, min2 = calibrate(count_fn, kinds, sel, anchor + origin, n, origin=origin)
    if rank < world - 1:
        clip = kinds == 2
        kinds = kinds.copy()
        kinds[clip] = 0
        max1 = max1.copy()
        max1[clip] = np.nextafter(np.float32(origin + SLAB), np.float32(-np.inf))
    return kinds, min1, max1, min2, sel


def query_fields(q, dt="f32"):
    """(kinds, min1, max1, min2) of a pst_query array, bounds in the value type."""
    t = {"f32": np.float32, "f64": np.float64, "i32": np.int32}[dt]
    sz = np.dtype(t).itemsize
    out = [np.asarray(q["kind"])]
    for f in ("min1", "max1", "min2"):
        raw = np.ascontiguousarray(q[f]).view(np.uint8).reshape(-1, 8)[:, :sz]
        out.append(np.ascontiguousarray(raw).view(t)[:, 0])
    return out


def gen_points_exp_device(n, seed, torch, mean_gap=0.01):
    """(n, 3) int32 tensor of PointStruct<float, uint32_t, 1> records of the
    batched-queries distribution: dim1 ~ U[0, 1), dim2 = dim1 + Exp(mean 0.01)
    (float32 add, rounded once), ids 0..n-1."""
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    d1 = torch.rand(n, generator=g, device="cuda", dtype=torch.float32)
    gap = torch.empty(n, device="cuda", dtype=torch.float32).exponential_(1.0 / mean_gap, generator=g)
    d2 = d1 + gap
    rec = torch.empty((n, 3), dtype=torch.int32, device="cuda")
    rec[:, 0] = d1.view(torch.int32)
    rec[:, 1] = d2.view(torch.int32)
    rec[:, 2] = torch.arange(n, device="cuda", dtype=torch.int32)
    del d1, d2, gap
    return rec


def gen_points_host(n, seed):
    rng = np.random.default_rng(seed)
    d1 = (rng.random(n, dtype=np.float32) * np.float32(1 << 24)).astype(np.float32)
    d2 = (d1 + rng.random(n, dtype=np.float32) * np.float32(1 << 16)).astype(np.float32)
    import oracle
    return oracle.make_points(d1, d2, np.arange(n, dtype=np.uint32), "f32")


def query_plan(nq, seed):
    rng = np.random.default_rng(seed)
    kinds = np.empty(nq, np.int32)
    kinds[: nq // 2] = 0
    kinds[nq // 2: 3 * nq // 4] = 1
    kinds[3 * nq // 4:] = 2
    rng.shuffle(kinds)
    sel = np.exp(rng.uniform(np.log(SEL_LO), np.log(SEL_HI), nq))
    anchor = rng.uniform(0, 1 << 24, nq)
    return kinds, sel, anchor


def calibrate(count_fn, kinds, sel, anchor, n, iters=24, domain=float(1 << 24), spread=float(1 << 16), origin=0.0):
    """Bisection of each query's free bound so that its exact count is ~sel * n,
    over brackets that keep every trial count within ~4x of the target (a trial
    never asks for a large fraction of the tree).  dim1 ~ U[0, domain) and
    dim2 - dim1 in [0, spread) (U[0, 2^16) for the large random trees; for the
    exponential gaps of the batched-queries distribution, a bound its largest gap
    stays below; a dim1 range that starts at `origin` shifts the brackets of the
    right queries with it):
      3-sided [a, a + W] with min2 = a: W free in [0, 4 s domain];
      left (b, c): dim2 bound c free in [b - 2 s domain - spread, b + spread];
      right (a, c): c free in [max(a, domain - 2 s domain - spread), domain + spread].
    count_fn(kinds, min1, max1, min2) -> exact counts."""
    nq = len(kinds)
    target = sel * n
    three, left, right = kinds == 0, kinds == 1, kinds == 2
    w = spread
    top = origin + domain
    lo = np.where(three, 0.0, np.where(left, anchor - 2 * sel * domain - w,
                                        np.maximum(anchor, top - 2 * sel * domain - w)))
    hi = np.where(three, 4 * sel * domain + 64 * domain / (1 << 24), np.where(left, anchor + w, top + w))
    best = (lo + hi) / 2
    best_err = np.full(nq, np.inf)

    def bounds(x):
        min1 = np.where(three | right, anchor, 0.0)
        max1 = np.where(three, anchor + x, np.where(left, anchor, 0.0))
        min2 = np.where(three, anchor, x)
        return min1.astype(np.float32), max1.astype(np.float32), min2.astype(np.float32)

    for _ in range(iters):
        mid = (lo + hi) / 2
        c = count_fn(kinds, *bounds(mid)).astype(np.float64)
        err = np.abs(c - target) / np.maximum(target, 1)
        upd = err < best_err
        best[upd] = mid[upd]
        best_err[upd] = err[upd]
        grow = np.where(three, c < target, c > target)  # move the free bound up
        lo = np.where(grow, mid, lo)
        hi = np.where(grow, hi, mid)
    return bounds(best)


def disjoint_plan(nq, seed, domain=float(1 << 24), origin=0.0):
    """nq 3-sided queries over consecutive, disjoint dim1 ranges that cover the whole
    domain, with min2 = the range's lower bound, so every point is reported by
    exactly one query (dim2 >= dim1 >= the bound): no point is read for two queries.
    Range widths are proportional to log-uniform weights on [1e-7, 1e-2], so the
    output sizes are as uneven as in the mixed plan.  Returns (kinds, min1, max1,
    min2) in float32."""
    rng = np.random.default_rng(seed)
    w = np.exp(rng.uniform(np.log(SEL_LO), np.log(SEL_HI), nq))
    edges = (origin + np.concatenate([[0.0], np.cumsum(w / w.sum())]) * domain).astype(np.float32)
    edges[0] = np.float32(-np.inf)
    a = edges[:-1]
    # each range ends just below where the next one starts (bounds are inclusive)
    b = np.nextafter(edges[1:], np.float32(-np.inf)).astype(np.float32)
    b[-1] = np.float32(np.inf)
    return np.zeros(nq, np.int32), a, b, a.copy()


def time_pass(eng, q_dev, out, offs, steps, warmup, stream, torch):
    """Mean device time (CUDA events on the launching stream) of `steps` batched
    passes over device-resident queries, after `warmup` untimed ones."""
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    for _ in range(warmup):
        eng.run(q_dev, out, offs, queries_on_device=True, sync=False)
    torch.cuda.synchronize()
    ms = []
    for _ in range(steps):
        ev[0].record(stream)
        eng.run(q_dev, out, offs, queries_on_device=True, sync=False)
        ev[1].record(stream)
        ev[1].synchronize()
        ms.append(ev[0].elapsed_time(ev[1]))
    return statistics.mean(ms)


def construct_roofline(n, ms, peak, peak_kind, val_bytes=4, id_bytes=4, key_bits=32, digit_bits=8):
    """Construction against HBM with the algorithmic bytes of the path's definition:
    the index sorts, ceil(key_bits / digit_bits) radix passes of n (key + u32 index)
    pairs read and written (16 B per point and pass for 4-byte keys), plus population,
    ceil(log2(n + 1)) levels of an index read and written per point and one write
    of every slot (three values, id, bitcode)."""
    levels = int(n).bit_length()
    slots = (1 << levels) - 1
    passes = -(-key_bits // digit_bits)
    sort_b = passes * n * 2 * (val_bytes + 4)
    pop_b = levels * 8 * n + slots * (3 * val_bytes + id_bytes + 1)
    ach = (sort_b + pop_b) / (ms / 1000.0) / 1e9
    return {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
            "traffic": None, "algorithmic_bytes": sort_b + pop_b, "sort_bytes": sort_b, "populate_bytes": pop_b,
            "peak_source": f"{peak_kind} hbm_gbs"}


def batched_queries_config(pst, torch, stream, steps, warmup, n=1 << 26, seed=3, plain_n=NQ):
    """The batched-queries configuration: one tree of 2^26 float32 points, dim1 ~
    U[0,1), dim2 = dim1 + Exp(mean 0.01); 4096 queries per pass (50 % 3-sided, 25 %
    left, 25 % right, selectivities log-uniform in [1e-7, 1e-2], bounds bisected on
    exact counts); the batched pass against the same 4096 queries as plain drop-in
    launches, one blocking call each."""
    rec = gen_points_exp_device(n, seed, torch)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    tree = pst.StaticPSTGPU(rec, n, "f32", True)
    torch.cuda.synchronize()
    build_ms = 1000 * (time.perf_counter() - t0)
    del rec
    eng = pst.BatchEngine(tree, max_queries=NQ, task_capacity=n >> 2)
    kinds, sel, anchor = query_plan(NQ, 9)
    anchor = anchor / float(1 << 24)

    def count_fn(k, a, b, c):
        return eng.count(pst.make_queries(k, a, b, c, "f32"))[0].cpu().numpy()
    min1, max1, min2 = calibrate(count_fn, kinds, sel, anchor, n, domain=1.0, spread=0.25)
    q_host = pst.make_queries(kinds, min1, max1, min2, "f32")
    _, total = eng.count(q_host)
    q_dev = torch.from_numpy(q_host.view(np.uint8).copy()).to("cuda")
    out = torch.empty(total * 4 + 16, dtype=torch.uint8, device="cuda")
    offs = torch.empty(NQ + 1, dtype=torch.int64, device="cuda")
    st, tot = eng.run(q_dev, out, offs, queries_on_device=True, sync=True)
    assert st == 0 and tot == total
    ms = time_pass(eng, q_dev, out, offs, steps, warmup, stream, torch)
    names = {0: "three", 1: "left", 2: "right"}
    m = min(plain_n, NQ)
    pst.free_device(tree.search_device(names[int(kinds[0])], min1[0], max1[0], min2[0])[0])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plain_pts = 0
    for i in range(m):
        ptr, c = tree.search_device(names[int(kinds[i])], min1[i], max1[i], min2[i])
        pst.free_device(ptr)
        plain_pts += c
    plain_s = time.perf_counter() - t0
    eng.close()
    tree.close()
    del out, q_dev
    torch.cuda.empty_cache()
    return {"workload": "batched-4096-mixed-queries-2^26-f32-exp", "n_points": n,
            "distribution": "dim1 ~ U[0,1), dim2 = dim1 + Exp(mean 0.01)", "queries_per_pass": NQ,
            "points_per_pass": int(total), "batched_ms": ms, "batched_pts_per_s": total / (ms / 1000.0),
            "batched_queries_per_s": NQ / (ms / 1000.0), "plain_queries": m, "plain_s": plain_s,
            "plain_queries_per_s": m / plain_s, "plain_points": int(plain_pts),
            "batched_vs_plain_qps": (NQ / (ms / 1000.0)) / (m / plain_s), "build_ms": build_ms,
            "bytes_per_pt": BYTES_PER_PT}


def blob_volume_device(px, py, pz, seed, torch, nblobs=32, noise=0.01):
    """Sum of 32 isotropic Gaussian blobs (centres uniform over the grid, sigma
    ~U[8,40] voxels, amplitude ~U[0.5,1]) + N(0, noise), float32 (pz, py, px) on
    the device; each blob is evaluated separably over its 4-sigma box."""
    rng = np.random.default_rng(seed)
    vol = torch.zeros((pz, py, px), dtype=torch.float32, device="cuda")
    for _ in range(nblobs):
        c = rng.uniform([0, 0, 0], [px, py, pz])
        s = rng.uniform(8.0, 40.0)
        a = float(rng.uniform(0.5, 1.0))
        lo = np.maximum(np.floor(c - 4 * s).astype(int), 0)
        hi = np.minimum(np.ceil(c + 4 * s).astype(int) + 1, [px, py, pz])
        g = [torch.exp(-0.5 * ((torch.arange(int(lo[i]), int(hi[i]), device="cuda", dtype=torch.float32)
                                 - float(c[i])) / s) ** 2) for i in range(3)]
        vol[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] += a * (g[2][:, None, None] * g[1][None, :, None]
                                                           * g[0][None, None, :])
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    if vol.numel() <= 1 << 30:
        vol += noise * torch.randn(vol.shape, generator=gen, device="cuda", dtype=torch.float32)
    else:
        # large volumes: the noise in z-slabs of at most 2^28 values, through one buffer
        per = max(1, (1 << 28) // (py * px))
        buf = torch.empty((per, py, px), device="cuda", dtype=torch.float32)
        for z0 in range(0, pz, per):
            z1 = min(pz, z0 + per)
            b = buf[: z1 - z0]
            b.normal_(generator=gen)
            vol[z0:z1].add_(b, alpha=noise)
        del buf
    return vol


# ---------------------------------------------------------------------------
# large random trees: every value type, kind and selectivity (run with --sweep)

SWEEP_TYPES = (("f32", True), ("f64", True), ("i32", True), ("f32", False))
SWEEP_SEL = (1e-5, 1e-3, 1e-1)
SWEEP_BATCH = 32


def gen_points_typed(n, seed, dt, has_id, torch):
    """PointStruct records of dim1 ~U[0,2^24), dim2 = dim1 + U[0,2^16) in the value type
    (integer-valued draws for i32), ids 0..n-1; returned as a byte tensor."""
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    if dt == "i32":
        d1 = torch.randint(0, 1 << 24, (n,), generator=g, device="cuda", dtype=torch.int32)
        d2 = d1 + torch.randint(0, 1 << 16, (n,), generator=g, device="cuda", dtype=torch.int32)
    else:
        tt = torch.float32 if dt == "f32" else torch.float64
        d1 = torch.rand(n, generator=g, device="cuda", dtype=tt) * float(1 << 24)
        d2 = d1 + torch.rand(n, generator=g, device="cuda", dtype=tt) * float(1 << 16)
    wide = dt == "f64"
    it = torch.int64 if wide else torch.int32
    rec = torch.zeros((n, 3 if has_id else 2), dtype=it, device="cuda")
    rec[:, 0] = d1.view(it)
    rec[:, 1] = d2.view(it)
    if has_id:
        rec[:, 2] = torch.arange(n, device="cuda", dtype=it)  # id in the low word, padding zero
    del d1, d2
    return rec


def ips_scan(pst, torch, pts, n, dt, has_id, reps=5):
    """Interval parallel search (the full-scan comparator) over n device points for a
    stabbing value in the middle of the dim1 domain: ms per call (device time between
    CUDA events, each call returning its count), hits, and GB/s of points read plus
    records written."""
    import ctypes as C
    lib = pst.lib()
    vs = 8 if dt == "f64" else 4
    v = (1 << 23) if dt == "i32" else float(1 << 23)
    ret = 0 if has_id else 1
    rec_bytes = 4 if has_id else 2 * vs
    cap = max(n // 16, 1)
    buf = torch.empty(cap * rec_bytes, dtype=torch.uint8, device="cuda")
    cnt = C.c_uint64()

    def call():
        pst.pst._check(lib.pst_ips_search_into(pst.pst.DTYPE[dt], 1 if has_id else 0, C.c_void_p(pts.data_ptr()), n,
                                               pst.pst.value_arg(dt, v), ret, C.c_void_p(buf.data_ptr()), cap,
                                               C.byref(cnt), None))
        return cnt.value
    for _ in range(2):
        call()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    torch.cuda.synchronize()
    ev[0].record()
    for _ in range(reps):
        k = call()
    ev[1].record()
    ev[1].synchronize()
    ms = ev[0].elapsed_time(ev[1]) / reps
    pt_bytes = pts.element_size() * pts.numel() // n
    return {"dtype": dt, "ids": has_id, "n": n, "v": v, "hits": k, "ms": ms,
            "gbs": (n * pt_bytes + k * rec_bytes) / (ms / 1000) / 1e9, "bytes_per_point": pt_bytes}


def sweep(pst, torch, n, peak, seed=1):
    """Per value type: build, then for each kind and selectivity a batch of 32 queries
    calibrated to s * n points each: batched pass time and one plain query; and one
    interval parallel search over the same points (returned as the "ips" rows)."""
    out, ips_rows = [], []
    rng = np.random.default_rng(seed)
    for dt, has_id in SWEEP_TYPES:
        vs = 8 if dt == "f64" else 4
        pts = gen_points_typed(n, seed, dt, has_id, torch)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        tree = pst.StaticPSTGPU(pts, n, dt, has_id)
        torch.cuda.synchronize()
        build_ms = 1000 * (time.perf_counter() - t0)
        r = ips_scan(pst, torch, pts, n, dt, has_id)
        # the scan's algorithmic bytes: dim1 and dim2 of every point, id and record of every hit
        vs_ = 8 if dt == "f64" else 4
        r["algorithmic_bytes"] = n * 2 * vs_ + r["hits"] * ((4 if has_id else 0) + (4 if has_id else 2 * vs_))
        r["frac"] = r["algorithmic_bytes"] / (r["ms"] / 1000) / 1e9 / peak
        # the records are read whole (the id sits between the values): bytes of the layout
        r["frac_layout"] = r["gbs"] / peak
        ips_rows.append(r)
        log(f"ips {dt}{'' if has_id else '-noid'}: {r['hits']} hits, {r['ms']:.3f} ms = {r['gbs']:.0f} GB/s")
        del pts
        torch.cuda.empty_cache()
        ret = "ids" if has_id else "points"
        rec_bytes = 4 if has_id else 2 * vs
        # read dim1, dim2 (+ id) per reported point, write the record
        bpp = 2 * vs + (4 if has_id else 0) + rec_bytes
        eng = pst.BatchEngine(tree, max_queries=SWEEP_BATCH)
        for kind in (0, 1, 2):
            for s in SWEEP_SEL:
                kinds = np.full(SWEEP_BATCH, kind, np.int32)
                anchor = rng.uniform(0, (1 << 24) * (1 - 4 * s), SWEEP_BATCH)
                sel = np.full(SWEEP_BATCH, s)

                def count_fn(k, a, b, c):
                    if dt == "i32":
                        a, b, c = (np.round(x).astype(np.int32) for x in (a, b, c))
                    counts, _ = eng.count(pst.make_queries(k, a, b, c, dt))
                    return counts.cpu().numpy()
                a, b, c = calibrate(count_fn, kinds, sel, anchor, n)
                if dt == "i32":
                    a, b, c = (np.round(x).astype(np.int32) for x in (a, b, c))
                q = pst.make_queries(kinds, a, b, c, dt)
                counts, total = eng.count(q)
                qd = torch.from_numpy(q.view(np.uint8).copy()).to("cuda")
                buf = torch.empty(total * rec_bytes + 16, dtype=torch.uint8, device="cuda")
                offs = torch.empty(SWEEP_BATCH + 1, dtype=torch.int64, device="cuda")
                for _ in range(3):
                    eng.run(qd, buf, offs, ret=ret, queries_on_device=True, sync=True)
                ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
                reps = 5
                ev[0].record()
                for _ in range(reps):
                    eng.run(qd, buf, offs, ret=ret, queries_on_device=True, sync=False)
                ev[1].record()
                ev[1].synchronize()
                ms = ev[0].elapsed_time(ev[1]) / reps
                # one plain drop-in query (callee-allocated result), wall clock
                name = {0: "three", 1: "left", 2: "right"}[kind]
                args = (float(a[0]), float(b[0]), float(c[0])) if dt != "i32" else (int(a[0]), int(b[0]), int(c[0]))
                pst.free_device(tree.search_device(name, *args, ret=ret)[0])
                torch.cuda.synchronize()
                t1 = time.perf_counter()
                ptr, k1 = tree.search_device(name, *args, ret=ret)
                pst.free_device(ptr)
                plain_s = time.perf_counter() - t1
                row = {"dtype": dt, "ids": has_id, "kind": name, "sel": s, "queries": SWEEP_BATCH,
                       "mean_points": total / SWEEP_BATCH, "batch_ms": ms, "pts_per_s": total / (ms / 1000),
                       "gbs": total * bpp / (ms / 1000) / 1e9, "frac": total * bpp / (ms / 1000) / 1e9 / peak,
                       "bytes_per_pt": bpp, "build_ms": build_ms,
                       "plain_query_ms": plain_s * 1000, "plain_pts_per_s": k1 / plain_s if plain_s else None}
                out.append(row)
                log(f"sweep {dt}{'' if has_id else '-noid'} {name:5s} s={s:g}: {total / SWEEP_BATCH:.3g} pts/query, "
                    f"batch {ms:.3f} ms = {row['pts_per_s']:.3g} pts/s ({row['gbs']:.0f} GB/s), "
                    f"plain {plain_s * 1000:.1f} ms")
                del buf, qd
        eng.close()
        tree.close()
        torch.cuda.empty_cache()
    return out, ips_rows


# ---------------------------------------------------------------------------
# isosurface pipeline (run with --isosurface)

def isosurface_bench(pst, torch, dims=(512, 512, 512), seed=1, peak=None):
    """512^3 float32 blob volume -> 4^3 metacells (128^3 points) -> tree; at 16
    isovalues 0.05 + 0.06 i: the active metacells by twoSidedLeftSearch(iso, iso)
    (batched and plain) and by the interval parallel search, then marching cubes
    over the active metacells.  Device times by CUDA events."""
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        ev[0].record()
        for _ in range(reps):
            r = fn()
        ev[1].record()
        ev[1].synchronize()
        return r, ev[0].elapsed_time(ev[1]) / reps

    vol = blob_volume_device(*dims, seed, torch).reshape(-1).contiguous()
    recs, n = timed(lambda: pst.formMetacellTags(vol, dims, (4, 4, 4), "f32", True))[0], None
    (recs, n), mc_ms = timed(lambda: pst.formMetacellTags(vol, dims, (4, 4, 4), "f32", True))
    # build time: median of five builds after a first one, each timed alone (the
    # previous tree is released outside the timed region; a build's allocations can
    # take many times its kernels on a shared machine, hence the median)
    pst.StaticPSTGPU(recs, n, "f32", True).close()
    bms = []
    for _ in range(5):
        torch.cuda.synchronize()
        ev[0].record()
        tree = pst.StaticPSTGPU(recs, n, "f32", True)
        ev[1].record()
        ev[1].synchronize()
        bms.append(ev[0].elapsed_time(ev[1]))
        if len(bms) < 5:
            tree.close()
    build_ms = statistics.median(bms)
    isos = [0.05 + 0.06 * i for i in range(16)]
    eng = pst.BatchEngine(tree, max_queries=16)
    q = pst.make_queries(np.full(16, 1, np.int32), np.zeros(16), np.array(isos), np.array(isos), "f32")
    offs, res = eng.search(q)
    qd = torch.from_numpy(q.view(np.uint8).copy()).to("cuda")
    out_d = torch.empty(max(len(res) * 4, 16), dtype=torch.uint8, device="cuda")
    offs_d = torch.empty(17, dtype=torch.int64, device="cuda")
    _, batch_ms = timed(lambda: eng.run(qd, out_d, offs_d, queries_on_device=True, sync=False))
    ips_buf = torch.empty(n * 4, dtype=torch.uint8, device="cuda")
    lib = pst.lib()

    def ips(iso32):
        cnt = C.c_uint64()
        pst.pst._check(lib.pst_ips_search_into(0, 1, C.c_void_p(recs.data_ptr()), n, pst.pst.value_arg("f32", iso32),
                                               0, C.c_void_p(ips_buf.data_ptr()), n, C.byref(cnt), None))
        return cnt.value
    rows = []
    tri_total, mc_total_ms = 0, 0.0
    for i, iso in enumerate(isos):
        iso32 = float(np.float32(iso))
        t0 = time.perf_counter()
        ptr, k = tree.search_device("left", 0.0, iso32, iso32)
        torch.cuda.synchronize()
        plain_ms = 1000 * (time.perf_counter() - t0)
        pst.free_device(ptr)
        ids = torch.from_numpy(np.ascontiguousarray(res[int(offs[i]):int(offs[i + 1])]).view(np.int32)).to("cuda")
        k_ips, ips_ms = timed(lambda: ips(iso32))
        assert k_ips == k
        tri, mc_ms_i = timed(lambda: pst.marchingCubes(vol, dims, (4, 4, 4), ids, iso32))
        tri_total += len(tri)
        mc_total_ms += mc_ms_i
        rows.append({"iso": iso32, "active_metacells": int(k), "plain_query_ms": plain_ms, "ips_ms": ips_ms,
                     "triangles": int(len(tri)), "marching_cubes_ms": mc_ms_i})
        del tri, ids
    mc_bytes = dims[0] * dims[1] * dims[2] * 4 + n * 12  # read the volume, write (min, max, id) per metacell
    out = {"volume": list(dims), "metacells": n, "form_metacells_ms": mc_ms,
           "form_metacells_roofline": {"bound": "hbm", "algorithmic_bytes": mc_bytes,
                                       "achieved": mc_bytes / (mc_ms / 1000) / 1e9, "peak": peak, "unit": "GB/s",
                                       "frac": mc_bytes / (mc_ms / 1000) / 1e9 / peak if peak else None},
           "build_ms": build_ms, "build_runs_ms": bms,
           "batched_16_isovalues_ms": batch_ms, "marching_cubes_triangles_per_s": tri_total / (mc_total_ms / 1000),
           "per_isovalue": rows}
    eng.close()
    tree.close()
    del vol, recs
    torch.cuda.empty_cache()
    return out


# Vertex grids of the 8 served volumes: 4^3 metacells give 2^16, 2^18, 2^20, 2^21,
# 2^23, 2^24, 2^25 and 2^27 metacells (the largest volume, 2048^3 float32, is 34 GB
# and is dropped once its metacells are formed).
SERVING_VOLUMES = [(256, 256, 64), (256, 256, 256), (512, 512, 256), (512, 512, 512), (1024, 1024, 512),
                   (1024, 1024, 1024), (2048, 2048, 512), (2048, 2048, 2048)]


def serving_bench(pst, torch, seconds=1.5, seed=11):
    """8 resident trees of 4^3 metacells (2^16 .. 2^27 points) from Gaussian-blob
    volumes; Poisson arrivals; 90% isovalue queries (iso, iso) with iso ~ U[0,1] and
    10% 3-sided range queries [a, a + w], w ~ U[0, 0.1], min2 = a.  A batch is
    admitted by its exact result bytes (from its count pass) into a 4 GiB result
    arena, or else into free HBM while 16 GiB stay free.  Latency runs from the
    scheduled arrival (open loop) to the result complete in device memory
    (`device`, at 1k, 10k and 100k qps) and to the result in host memory (`host`,
    at 1k and 10k qps: at 100k qps the offered results, ~240 GB/s of ids, are far
    beyond the host link, so the queue only grows)."""
    trees = []
    for i, (px, py, pz) in enumerate(SERVING_VOLUMES):
        vol = blob_volume_device(px, py, pz, seed + i, torch)
        mc, n = pst.formMetacellTags(vol.reshape(-1), (px, py, pz), (4, 4, 4), "f32", True)
        del vol
        torch.cuda.empty_cache()
        trees.append(pst.StaticPSTGPU(mc, n, "f32", True))
        del mc
    torch.cuda.empty_cache()
    out = {"trees_points": [t.n for t in trees]}
    for mode, keep, rates in (("device", 0, (1000, 10000, 100000)), ("host", 2, (1000, 10000))):
        srv = pst.Server(max_batch=1024, slots_per_tree=2, out_budget_bytes=4 << 30, keep_results=keep,
                         hbm_headroom_bytes=16 << 30)
        idx = [srv.add_tree(t) for t in trees]
        rng = np.random.default_rng(seed)
        res = {}
        for rate in rates:
            n = int(rate * seconds)
            gaps = rng.exponential(1.0 / rate, n)
            tree_of = np.asarray(idx, np.uint32)[rng.integers(0, len(trees), n)]
            three = rng.random(n) < 0.1
            a = rng.uniform(0, 1, n).astype(np.float32)
            w = rng.uniform(0, 0.1, n).astype(np.float32)
            kinds = np.where(three, 0, 1).astype(np.int32)
            q = pst.make_queries(kinds, np.where(three, a, 0), np.where(three, a + w, a), a, "f32")
            srv.reset_stats()
            t0 = time.monotonic_ns() + 2_000_000
            arrive = t0 + np.cumsum(gaps * 1e9).astype(np.uint64)
            k = 0
            while k < n:
                now = time.monotonic_ns()
                j = int(np.searchsorted(arrive, now, side="right"))
                if j > k:
                    srv.submit(tree_of[k:j], q[k:j], arrival_ns=arrive[k:j])
                    k = j
                else:
                    time.sleep(20e-6)
            srv.drain(120000)
            st = srv.stats()
            res[f"{rate}qps"] = {"p50_ms": st["p50_ms"], "p90_ms": st["p90_ms"], "p99_ms": st["p99_ms"],
                                 "mean_ms": st["mean_ms"], "completed": st["completed"], "failed": st["failed"],
                                 "batches": st["batches"], "points": st["points"], "spilled_batches": st["spilled"],
                                 "peak_arena_bytes": st["peak_out_bytes"],
                                 "throughput_qps": st["completed"] / st["busy_s"] if st["busy_s"] else None,
                                 "worker_cpu_s": st["worker_cpu_s"],
                                 "worker_cpu_share": st["worker_cpu_s"] / st["busy_s"] if st["busy_s"] else None}
        srv.close()
        out[mode] = res
    for t in trees:
        t.close()
    return out


# ---------------------------------------------------------------------------
# clocks

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index=0):
        self.samples = []
        self.proc = None
        self.dev = device_index

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for nm, v in zip(names, s[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


# ---------------------------------------------------------------------------
# CPU reference (the reference's StaticPSTCPUIter, compiled from its sources)

_REF_CACHE = {}


def reference_sample(n_sample, nq_sample, seed=1):
    """The reference's StaticPSTCPUIter built over a sample of the workload and
    queries of the same kind mix and selectivities, calibrated once with the
    oracle's brute-force counts (threaded C scans, not timed)."""
    key = (n_sample, nq_sample, seed)
    if key in _REF_CACHE:
        return _REF_CACHE[key]
    import oracle
    from concurrent.futures import ThreadPoolExecutor
    pts = gen_points_host(n_sample, seed)
    t0 = time.perf_counter()
    ref = oracle.Ref(pts, "f32")
    build_s = time.perf_counter() - t0
    kinds, sel, anchor = query_plan(nq_sample, seed + 1)
    names = {0: "three", 1: "left", 2: "right"}

    def count_fn(k, a, b, c):
        def one(i):
            return len(oracle.Orc.brute(pts, "f32", names[int(k[i])], a[i], b[i], c[i]))
        with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
            return np.array(list(ex.map(one, range(len(k)))), np.int64)
    min1, max1, min2 = calibrate(count_fn, kinds, sel, anchor, n_sample, iters=16)
    qs = [(names[int(kinds[i])], float(min1[i]), float(max1[i]), float(min2[i])) for i in range(nq_sample)]
    _REF_CACHE[key] = (ref, qs, build_s)
    return _REF_CACHE[key]


def cpu_reference_time(ref, qs, threads):
    """One timed pass of the reference's searches over qs; returns (pts/s, q/s, s, pts)."""
    from concurrent.futures import ThreadPoolExecutor
    t0 = time.perf_counter()
    if threads == 1:
        counts = [ref.count(*q) for q in qs]
    else:
        with ThreadPoolExecutor(max_workers=threads) as ex:
            counts = list(ex.map(lambda q: ref.count(*q), qs))
    dt = time.perf_counter() - t0
    total = int(sum(counts))
    return total / dt, len(qs) / dt, dt, total


def ref_kind():
    import oracle
    return "reference" if oracle.Ref.available() else "port"


# ---------------------------------------------------------------------------

def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle
    if not oracle.Ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libpstref.so was not built"}))
        return 0
    threads = os.cpu_count() or 1
    n_sample, nq_sample = 1 << 22, 512
    ref, qs, build_s = reference_sample(n_sample, nq_sample)
    # Each reference search allocates a result array of n records (new[]), and
    # those allocations contend across threads; use whichever of one thread or
    # all host threads is faster on this box.
    t_one = cpu_reference_time(ref, qs[:64], 1)[0]
    t_all = cpu_reference_time(ref, qs[:64], threads)[0]
    if t_one > t_all:
        threads = 1
    vals = []
    for i in range(args.warmup + args.steps):
        v, qps, dt, tot = cpu_reference_time(ref, qs, threads)
        if i >= args.warmup:
            vals.append((v, qps, {"search_s": dt}))
    info0 = {"build_s": build_s}
    v = statistics.median(x[0] for x in vals)
    qps = statistics.median(x[1] for x in vals)
    sample = (f"StaticPSTCPUIter over a 2^22-point sample of the workload, {nq_sample} queries per step "
              f"with the same kind mix and selectivities, {threads} thread(s) (faster of 1 and all {os.cpu_count()})")
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * statistics.median(x[2]["search_s"] for x in vals),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "queries_per_s": qps,
            "config": {"workload": "batched-4096-mixed-queries-2^28-f32 (reference CPU sample)", "n_points": N_POINTS,
                       "queries_per_step": NQ, "selectivity": [SEL_LO, SEL_HI]},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample,
                             "build_s_sample": info0["build_s"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200")
    ap.add_argument("--points-log2", type=int, default=28)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the 2^26 batched-queries configuration")
    ap.add_argument("--no-tune", action="store_true", help="the default launch shape instead of the autotuner's")
    ap.add_argument("--shape", default=None,
                    help="a launch shape as JSON (block_threads, blocks_per_sm, emit_records, top_pass_queries) "
                         "instead of tuning, e.g. to profile the shape a tuned run chose")
    ap.add_argument("--plain-queries", type=int, default=256)
    ap.add_argument("--no-sweep", action="store_true", help="skip the large-random-tree matrix (every value type x "
                                                              "kind x selectivity, and the interval scans)")
    ap.add_argument("--no-isosurface", action="store_true", help="skip the 512^3 isosurface pipeline")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    pst = load_package()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    # one GPU per rank (LOCAL_RANK); a box with fewer GPUs than ranks runs several
    # ranks per GPU, which only a functional check of the N > 1 path should do
    torch.cuda.set_device(local % max(torch.cuda.device_count(), 1))
    dist = None
    cdev = "cuda"  # device of the collectives' tensors
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = os.environ.get("PST_BENCH_DIST_BACKEND", "nccl")  # gloo: the functional check
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        cdev = "cuda" if backend == "nccl" else "cpu"
    n = 1 << args.points_log2
    stream = torch.cuda.current_stream()

    # ---- construction (timed separately, reported as extra keys)
    pts_d = slab_points_device(n, rank, torch)
    bounds = slab_bounds(pts_d, torch)
    torch.cuda.synchronize()
    c0 = time.perf_counter()
    tree = pst.StaticPSTGPU(pts_d, n, "f32", True)  # first build: allocator and module warm-up
    torch.cuda.synchronize()
    construct_cold_ms = 1000 * (time.perf_counter() - c0)
    tree.close()
    # the median of nine warm builds: a build's wall time includes the allocation
    # of the tree and of its working set (7.1 GiB and more at 2^28), whose cost
    # varies from call to call (single builds of several times the median were seen
    # on shared machines) while the kernels do not (NVTX range "construct" around
    # the last build only)
    construct_runs = []
    n_builds = 9
    for b in range(n_builds):
        c0 = time.perf_counter()
        if b == n_builds - 1:
            torch.cuda.nvtx.range_push("construct")
        tree = pst.StaticPSTGPU(pts_d, n, "f32", True)
        if b == n_builds - 1:
            torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        construct_runs.append(1000 * (time.perf_counter() - c0))
        if b < n_builds - 1:
            tree.close()
    construct_ms = statistics.median(construct_runs)
    log(f"constructed 2^{args.points_log2} points in {construct_ms:.1f} ms (median of "
        f"{', '.join(f'{x:.1f}' for x in construct_runs)}; first build {construct_cold_ms:.1f} ms)")
    del pts_d
    torch.cuda.empty_cache()

    # ---- queries: this shard's block of the global list (bisected on its own
    # counts); with several shards every rank routes the whole list by the shards'
    # bounds and runs the queries that can meet its slab
    eng = pst.BatchEngine(tree, max_queries=NQ, task_capacity=max(1 << 20, n >> 2))

    def count_fn(k, a, b, c):
        q = pst.make_queries(k, a, b, c, "f32")
        counts, _ = eng.count(q)
        return counts.cpu().numpy()
    kinds, min1, max1, min2, sel = sharded_block(count_fn, rank, world, n)
    log("calibrated query bounds")
    q_host = pst.make_queries(kinds, min1, max1, min2, "f32")
    routed_n = NQ
    if world > 1:
        import importlib.util as _ilu
        _spec = _ilu.spec_from_file_location("pst_sharded", PKG_DIR / "sharded.py")
        sharded = _ilu.module_from_spec(_spec)
        _spec.loader.exec_module(sharded)
        qb = torch.from_numpy(q_host.view(np.uint8).copy()).to(cdev)
        blocks = [torch.empty_like(qb) for _ in range(world)]
        dist.all_gather(blocks, qb)
        rb = [torch.zeros(4, dtype=torch.float64, device=cdev) for _ in range(world)]
        dist.all_gather(rb, torch.tensor(bounds, dtype=torch.float64, device=cdev))
        ranges = torch.stack(rb).cpu().numpy()
        q_all = torch.cat(blocks).cpu().numpy().view(pst.pst.QUERY_NP)
        ak, a1, a2, a3 = query_fields(q_all)
        routed = np.nonzero(sharded.route_many(ak, a1, a2, a3, ranges)[:, rank])[0]
        q_host = np.ascontiguousarray(q_all[routed])
        kinds, min1, max1, min2 = query_fields(q_host)
        routed_n = len(routed)
        log(f"shard {rank}: {routed_n} of {world * NQ} queries routed here")
    # ---- launch shape: the project's autotuner times its candidates on these
    # queries (not cached across runs: every box times them afresh)
    tuned = None
    if args.shape:
        tuned = dict(json.loads(args.shape), ms=None, default_ms=None, tried=[])
    elif not args.no_tune:
        import importlib
        autotune = importlib.import_module("pst_b200.autotune")
        tuned = autotune.tune(tree, q_host, repeats=5, cache_path=None, task_capacity=max(1 << 20, n >> 2))
        dflt = [ms for sh, ms in tuned["tried"] if sh["block_threads"] == 256 and sh["blocks_per_sm"] == 0
                and sh["emit_records"] == 8]
        tuned["default_ms"] = dflt[0] if dflt else None
        for sh, ms in tuned["tried"]:
            log("  shape " + " ".join(f"{k}={sh[k]}" for k in pst.pst.TUNING_FIELDS) + f": {ms:.3f} ms")
        log("autotuned launch shape: " + ", ".join(f"{k}={tuned[k]}" for k in pst.pst.TUNING_FIELDS) +
            f" ({tuned['ms']:.3f} ms per pass; default shape {tuned['default_ms']:.3f} ms)")
    eng.close()
    eng = pst.BatchEngine(tree, max_queries=max(routed_n, NQ), task_capacity=max(1 << 20, n >> 2), tuning=tuned)
    counts, total = eng.count(q_host)
    q_dev = torch.from_numpy(q_host.view(np.uint8).copy()).to("cuda")
    out = torch.empty(total * 4 + 16, dtype=torch.uint8, device="cuda")
    offs = torch.empty(max(routed_n, NQ) + 1, dtype=torch.int64, device="cuda")
    st, tot = eng.run(q_dev, out, offs, queries_on_device=True, sync=True)
    assert st == 0 and tot == total
    frontier = eng.last_stats()
    log(f"frontier: {frontier['records']} alive records ({total / max(frontier['records'], 1):.1f} points each), "
        f"{frontier['seeds']} seeds, {frontier['boundary']} boundary nodes; per level {frontier['per_level']}")

    # ---- device-resident timing (value)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    for _ in range(args.warmup):
        eng.run(q_dev, out, offs, queries_on_device=True, sync=False)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    step_ms = []
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("timed")
        for _ in range(args.steps):
            ev[0].record(stream)
            eng.run(q_dev, out, offs, queries_on_device=True, sync=False)
            ev[1].record(stream)
            ev[1].synchronize()
            step_ms.append(ev[0].elapsed_time(ev[1]))
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
    st_, tot2 = eng.run(q_dev, out, offs, queries_on_device=True, sync=True)
    assert st_ == 0 and tot2 == total
    my_ms = statistics.mean(step_ms)
    log(f"timed {args.steps} steps: {my_ms:.3f} ms/step, {total} points/step")
    pts_all, ms_all = float(total), my_ms
    if dist:
        t = torch.tensor([my_ms], device=cdev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_all = float(t.item())
        p = torch.tensor([float(total)], device=cdev, dtype=torch.float64)
        dist.all_reduce(p, op=dist.ReduceOp.SUM)
        pts_all = float(p.item())
    value = pts_all / (ms_all / 1000.0)
    qps = world * NQ / (ms_all / 1000.0)

    # ---- end to end through the public call with host buffers
    q_pin = torch.from_numpy(q_host.view(np.uint8).copy()).pin_memory()
    out_pin = torch.empty(total * 4 + 16, dtype=torch.uint8).pin_memory()
    offs_pin = torch.empty(offs.numel(), dtype=torch.int64).pin_memory()
    e2e_ms = []
    for i in range(args.warmup + max(3, args.steps // 4)):
        torch.cuda.synchronize()
        ev[0].record(stream)
        q_dev.copy_(q_pin, non_blocking=True)
        eng.run(q_dev, out, offs, queries_on_device=True, sync=True)
        out_pin.copy_(out, non_blocking=True)
        offs_pin.copy_(offs, non_blocking=True)
        ev[1].record(stream)
        ev[1].synchronize()
        if i >= args.warmup:
            e2e_ms.append(ev[0].elapsed_time(ev[1]))
    e2e_mean = statistics.mean(e2e_ms)
    if dist:
        t = torch.tensor([e2e_mean], device=cdev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_mean = float(t.item())
    e2e_val = pts_all / (e2e_mean / 1000.0)
    log(f"e2e {e2e_mean:.3f} ms/step")

    # ---- plain per-query drop-in path on a sample of the same queries: the blocking
    # call that hands back a device array of exactly `count` ids (as the reference's
    # searches do), released after each call
    plain_n = min(args.plain_queries, len(q_host))
    names = {0: "three", 1: "left", 2: "right"}
    ptr, _ = tree.search_device(names[int(kinds[0])], float(min1[0]), float(max1[0]), float(min2[0]))
    pst.free_device(ptr)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plain_pts = 0
    for i in range(plain_n):
        ptr, cnt = tree.search_device(names[int(kinds[i])], float(min1[i]), float(max1[i]), float(min2[i]))
        pst.free_device(ptr)
        plain_pts += cnt
    plain_s = time.perf_counter() - t0
    plain_qps = plain_n / plain_s
    log(f"plain per-query path: {plain_qps:.1f} queries/s")

    # ---- the same tree, queries over disjoint dim1 ranges: every point reported
    # exactly once per pass, so no row is read for two queries (no L2 reuse between
    # queries); the pass's HBM efficiency without overlap
    dk, da, db, dc = disjoint_plan(NQ, 13, origin=float(rank) * SLAB)  # this shard's slab
    dq_host = pst.make_queries(dk, da, db, dc, "f32")
    dq_dev = torch.from_numpy(dq_host.view(np.uint8).copy()).to("cuda")
    st_d, tot_d = eng.run(dq_dev, out, offs, queries_on_device=True, sync=True)
    assert st_d == 0 and tot_d == n, (st_d, tot_d)  # each point exactly once
    torch.cuda.nvtx.range_push("disjoint")
    dis_ms = time_pass(eng, dq_dev, out, offs, max(3, args.steps // 2), args.warmup, stream, torch)
    torch.cuda.nvtx.range_pop()
    log(f"disjoint ranges: {dis_ms:.3f} ms/pass for {tot_d} points")

    # ---- roofline of the batched search pass
    peak, peak_kind = measured_peak()
    achieved = total * BYTES_PER_PT / (my_ms / 1000.0) / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": None, "kernel": "batched search pass (k_bfs_level x levels + scan + k_emit)",
            "bytes_per_unit": BYTES_PER_PT, "units_per_launch": total, "peak_source": f"{peak_kind} hbm_gbs",
            "frac_at_min_bytes": total * BYTES_PER_PT_MIN / (my_ms / 1000.0) / 1e9 / peak,
            "min_bytes_per_unit": BYTES_PER_PT_MIN}
    dis_ach = tot_d * BYTES_PER_PT / (dis_ms / 1000.0) / 1e9
    disjoint = {"workload": "batched-4096-disjoint-3-sided-2^28-f32", "points_per_pass": int(tot_d),
                "ms_per_pass": dis_ms, "pts_per_s": tot_d / (dis_ms / 1000.0),
                "roofline": {"bound": "hbm", "achieved": dis_ach, "peak": peak, "unit": "GB/s",
                             "frac": dis_ach / peak, "traffic": None, "bytes_per_unit": BYTES_PER_PT,
                             "units_per_launch": int(tot_d),
                             "frac_at_min_bytes": tot_d * BYTES_PER_PT_MIN / (dis_ms / 1000.0) / 1e9 / peak,
                             "peak_source": f"{peak_kind} hbm_gbs"}}
    prof = ROOT / "profiles" / "search_traffic.json"
    if prof.exists() and n == N_POINTS:
        try:
            tr = json.loads(prof.read_text())
            roof["traffic"] = tr["search_bytes_per_step"]
            roof["traffic_source"] = f"ncu dram bytes on {tr['measured_on']}, scaled to {tr['scaled_to']}"
            if "disjoint_bytes_per_pass" in tr:
                disjoint["roofline"]["traffic"] = tr["disjoint_bytes_per_pass"]
                disjoint["roofline"]["traffic_source"] = tr["disjoint_source"]
        except Exception:
            pass
    del dq_dev

    batched_cfg = None
    if rank == 0 and not args.no_extra:
        batched_cfg = batched_queries_config(pst, torch, stream, max(3, args.steps // 2), args.warmup)
        log("batched-queries configuration (2^26, exponential gaps): {:.3f} ms/pass, {:.3g} pts/s, "
            "{:.0f}x the plain launches in queries/s".format(batched_cfg["batched_ms"], batched_cfg["batched_pts_per_s"],
                                                            batched_cfg["batched_vs_plain_qps"]))

    levels_main = tree.info()["levels"]
    sweep_rows = ips_rows = None
    if rank == 0 and not args.no_sweep:
        # the large random trees need the device to themselves
        eng.close()
        tree.close()
        eng = tree = None
        torch.cuda.empty_cache()
        try:
            sweep_rows, ips_rows = sweep(pst, torch, n, peak)
        except Exception as e:  # an extra table must never sink the headline
            sweep_rows = {"error": str(e)}

    iso_res = None
    if rank == 0 and not args.no_isosurface:
        try:
            iso_res = isosurface_bench(pst, torch, peak=peak)
            log("isosurface: metacells {:.2f} ms, build {:.2f} ms, 16 isovalues batched {:.3f} ms, "
                "marching cubes {:.3g} triangles/s".format(iso_res["form_metacells_ms"], iso_res["build_ms"],
                                                         iso_res["batched_16_isovalues_ms"],
                                                         iso_res["marching_cubes_triangles_per_s"]))
        except Exception as e:
            iso_res = {"error": str(e)}

    serving = None
    if rank == 0 and not args.no_serving:
        try:
            serving = serving_bench(pst, torch)
            for mode in ("device", "host"):
                log(f"serving ({mode}): " + ", ".join(f"{k} p50 {v['p50_ms']:.2f} p99 {v['p99_ms']:.2f} ms"
                                                      for k, v in serving[mode].items()))
        except Exception as e:
            serving = {"error": str(e)}

    cpu = None
    if rank == 0 and not args.no_cpu:
        try:
            ref, qs, build_s = reference_sample(1 << 22, 128)
            v, q, dt, tot = cpu_reference_time(ref, qs, 1)
            cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": ref_kind(),
                   "sample": "StaticPSTCPUIter, 2^22-point sample tree of the same distribution, 128 queries of the "
                             "same kind mix and selectivities, 1 thread", "queries_per_s": q,
                   "build_s_sample": build_s}
        except Exception as e:  # the baseline must never sink the GPU number
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": ref_kind(), "sample": f"failed: {e}"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_all, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "batched-4096-mixed-queries-2^28-f32", "n_points": n, "ids": "u32",
                           "queries_per_step": NQ, "mix": "50% three / 25% left / 25% right",
                           "selectivity": [SEL_LO, SEL_HI], "results": "ids",
                           "l2": "inputs larger than L2 (tree 7.1 GiB)", "parallelism": (f"{world} dim1 shards of one point set (weak scaling: 2^28 points "
                                           f"and a block of 4096 queries per shard, every query routed to the "
                                           f"shards its bounds meet; no data-path collective)"
                                           if world > 1 else "one shard")},
                "routed_queries": routed_n,
                "autotune": None if tuned is None else {
                    "chosen": {k: tuned[k] for k in pst.pst.TUNING_FIELDS}, "ms": tuned["ms"],
                    "default_shape_ms": tuned["default_ms"], "candidates": len(tuned["tried"])},
                "queries_per_s": qps, "points_per_step": total,
                "frontier": {k: frontier[k] for k in ("records", "seeds", "boundary")},
                "plain_queries_per_s": plain_qps, "batched_vs_plain_qps": qps / world / plain_qps,
                "construct_ms": construct_ms, "construct_first_ms": construct_cold_ms, "construct_pts_per_s": n / (construct_ms / 1000.0),
                "construct": {"ms": construct_ms, "points": n, "runs_ms": construct_runs,
                              "roofline": construct_roofline(n, construct_ms, peak, peak_kind)},
                "disjoint": disjoint, "batched_queries_config": batched_cfg,
                "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": int(q_host.nbytes),
                        "d2h_bytes_per_step": int(total * 4 + offs.numel() * 8)},
                "gpu_launches": None, "roofline": roof, "cpu_baseline": cpu, "clocks": clk.summary(),
                "serving": serving}
        if sweep_rows is not None:
            line["sweep"] = sweep_rows
            line["ips"] = ips_rows
        if iso_res is not None:
            line["isosurface"] = iso_res
        # per step: the control block's load, query preparation, one kernel per level,
        # offsets, emit (a batch of 4096 queries takes the one-launch offsets scan)
        line["gpu_launches"] = (levels_main + 4) * args.steps
        print(json.dumps(line))
    if eng is not None:
        eng.close()
    if tree is not None:
        tree.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
