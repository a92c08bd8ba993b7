"""Batched mixed-codec decoding: batch construction, task tables, launches.

A batch is a list of items, each one column segment encoded with one codec
(its own container).  The planner turns items into warp-sized tasks
(gd_task, include/gd.h): one per brle chunk, per RLE v1 / RLE v2 lane stream,
per LZSS chunk and per Deflate stream, lays every payload and every output
into device arenas, and launches gd_batch_decode.  The task order given to
the launch is the scheduling decision: identity (static mapping task i ->
warp i mod W, the fallback), or longest-predicted-first through the dynamic
work queue (LPT list scheduling) with costs from the learned model
(compression_b200.costmodel) or from any other estimate.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import codecs as cc
from ._lib import lib

CODECS = ["brle", "rlev1", "rlev2", "lzss", "deflate"]
CODEC_ID = {c: i for i, c in enumerate(CODECS)}
# size granule of an item per codec: RLE v1 chunks are multiples of 32 lanes x
# COMP_COL_LEN (128 B); RLE v2 of 256 x READ_UNIT (32); LZSS of 128 B
GRANULE = {"brle": 16, "rlev1": 4096, "rlev2": 8192, "lzss": 128, "deflate": 16}
DEFAULT_CHUNK = {"brle": 256 * 1024, "rlev1": 128 * 1024, "rlev2": 256 * 1024, "lzss": 64 * 1024}

TASK_DTYPE = np.dtype([
    ("codec", "<u4"), ("param", "<u4"), ("lane", "<u4"), ("reserved", "<u4"),
    ("src", "<u8"), ("src_len", "<u8"), ("dst", "<u8"), ("dst_len", "<u8"),
    ("chunk_size", "<u8"), ("col_len", "<u8"), ("col_map", "<u8")])
assert TASK_DTYPE.itemsize == 72


@dataclass
class Item:
    codec: str
    raw: np.ndarray          # the decompressed bytes (uint8 view)
    enc: cc.Encoded


def _gen(codec: str, seed: int, nbytes: int) -> np.ndarray:
    if codec == "brle":
        return cc.gen_brle_bytes(seed, nbytes)
    if codec == "rlev1":
        return cc.gen_rlev1_ints(seed, nbytes // 4).view(np.uint8)
    if codec == "rlev2":
        return cc.gen_rlev2_ints(seed, nbytes // 8).view(np.uint8)
    return cc.gen_markov_copy(seed, nbytes, 4096 if codec == "lzss" else 32768)


def encode_item(codec: str, raw: np.ndarray, seed: int = 0) -> cc.Encoded:
    n = raw.size
    if codec == "brle":
        return cc.brle_encode(raw, min(DEFAULT_CHUNK["brle"], max(16, n)))
    if codec == "rlev1":
        return cc.rlev1_encode(raw, min(DEFAULT_CHUNK["rlev1"], n), 128, 4)
    if codec == "rlev2":
        return cc.rlev2_encode(raw, min(DEFAULT_CHUNK["rlev2"], n), 32)
    if codec == "lzss":
        return cc.lzss_encode(raw, min(DEFAULT_CHUNK["lzss"], n))
    # ~3% of Deflate streams use fixed or stored blocks
    r = (seed * 2654435761 % 1000) / 1000.0
    mode = np.array([1 if r < 0.015 else (2 if r < 0.03 else 0)], np.uint8)
    return cc.deflate_encode(raw, np.array([0, n], np.uint64), 6, mode, 1)


def make_mixed_batch(seed: int, n_items: int, total_bytes: int, lo: int = 4096, hi: int = 2 << 20,
                     mix=(0.20, 0.20, 0.10, 0.25, 0.25)) -> list[Item]:
    """Items with sizes log-uniform in [lo, hi] scaled to total_bytes, codecs
    RLE v1 / RLE v2 / byte-RLE / LZSS / Deflate in the proportions `mix`."""
    sizes = cc.loguniform_sizes(seed, n_items, lo, hi, total_bytes, 16)
    rng = np.random.default_rng(seed)
    order = ["rlev1", "rlev2", "brle", "lzss", "deflate"]
    counts = np.floor(np.array(mix) * n_items).astype(int)
    counts[-1] = n_items - counts[:-1].sum()
    codecs = np.concatenate([[order[i]] * counts[i] for i in range(5)])
    rng.shuffle(codecs)
    def one(i):
        codec, sz = codecs[i], sizes[i]
        g = GRANULE[codec]
        n = max(g, int(sz) // g * g)
        raw = _gen(codec, seed * 100003 + i, n)
        return Item(codec, raw, encode_item(codec, raw, seed * 7 + i))

    # items are independent: built on all host threads (the C ABI calls
    # release the interpreter lock); the result does not depend on the order
    import concurrent.futures as cf
    import os
    with cf.ThreadPoolExecutor(os.cpu_count() or 1) as ex:
        return list(ex.map(one, range(n_items)))


@dataclass
class Plan:
    """Device-resident batch: arenas, task table, per-item output views."""
    items: list
    tasks: np.ndarray                # TASK_DTYPE records (host copy, device addresses)
    task_item: np.ndarray            # item index of every task
    d_tasks: object = None
    d_in: object = None
    d_meta: object = None
    d_out: object = None
    out_off: np.ndarray = None       # byte offset of each item's output in d_out
    out_len: np.ndarray = None
    max_lane: int = 0
    d_status: object = None
    d_timing: object = None
    d_counter: object = None
    extra: dict = field(default_factory=dict)


def _align(x: int, a: int = 256) -> int:
    return (x + a - 1) // a * a


def build_plan(items: list[Item], device="cuda") -> Plan:
    import torch
    dev = torch.device(device)
    # ---- input arena (payloads) and metadata arena (col_len / col_map) ----
    in_off, pos = [], 0
    for it in items:
        in_off.append(pos)
        pos = _align(pos + it.enc.data.size + 16)
    h_in = np.zeros(max(pos, 256), np.uint8)
    for it, o in zip(items, in_off):
        h_in[o:o + it.enc.data.size] = it.enc.data
    meta_off, mpos = [], 0
    for it in items:
        meta_off.append(mpos)
        if "col_len" in it.enc.meta:
            mpos = _align(mpos + it.enc.meta["col_len"].nbytes + it.enc.meta.get("col_map", np.zeros(0)).nbytes)
    h_meta = np.zeros(max(mpos, 256), np.uint8)
    for it, o in zip(items, meta_off):
        if "col_len" in it.enc.meta:
            cl = it.enc.meta["col_len"].view(np.uint8)
            h_meta[o:o + cl.size] = cl
            if "col_map" in it.enc.meta:
                cm = it.enc.meta["col_map"]
                h_meta[o + cl.size:o + cl.size + cm.size] = cm
    # ---- output arena ----
    out_off, out_len, opos = [], [], 0
    for it in items:
        e = it.enc
        need = e.n_chunks * e.chunk_size if it.codec == "lzss" else e.n_out
        out_off.append(opos)
        out_len.append(e.n_out)
        opos = _align(opos + need + 16)
    d_in = torch.from_numpy(h_in).to(dev)
    d_meta = torch.from_numpy(h_meta).to(dev)
    d_out = torch.zeros(max(opos, 256), dtype=torch.uint8, device=dev)
    bi, bm, bo = d_in.data_ptr(), d_meta.data_ptr(), d_out.data_ptr()
    # ---- tasks ----
    recs, titem, tchunk = [], [], []
    max_lane = 0
    for ii, (it, io, mo, oo) in enumerate(zip(items, in_off, meta_off, out_off)):
        e, c = it.enc, it.codec
        if c == "brle":
            p = e.meta["ptr"]
            for k in range(e.n_chunks):
                recs.append((0, 0, 0, 0, bi + io + int(p[k]), int(p[k + 1] - p[k]), bo + oo + k * e.chunk_size,
                             min(e.chunk_size, e.n_out - k * e.chunk_size), e.chunk_size, 0, 0))
                titem.append(ii)
                tchunk.append(k)
        elif c in ("rlev1", "rlev2"):
            bo_ = e.meta["blk_off"]
            max_lane = max(max_lane, int(e.meta["col_len"].max()))
            param = (4 << 16) | 32 if c == "rlev1" else e.params["read_unit"]
            for k in range(e.n_chunks):
                for t in range(32):
                    recs.append((CODEC_ID[c], param, t, 0, bi + io + int(bo_[k]), int(bo_[k + 1] - bo_[k]),
                                 bo + oo + k * e.chunk_size, min(e.chunk_size, e.n_out - k * e.chunk_size),
                                 e.chunk_size, bm + mo + 8 * 32 * k, 0))
                    titem.append(ii)
                    tchunk.append(k)
        elif c == "lzss":
            bo_ = e.meta["blk_off"]
            ncl = e.meta["col_len"].nbytes
            for k in range(e.n_chunks):
                recs.append((3, 0, 0, 0, bi + io + int(bo_[k]), int(bo_[k + 1] - bo_[k]), bo + oo + k * e.chunk_size,
                             e.chunk_size, e.chunk_size, bm + mo + 8 * 32 * k, bm + mo + ncl + 32 * k))
                titem.append(ii)
                tchunk.append(k)
        else:
            recs.append((4, e.params["zlib_header"], 0, 0, bi + io + int(e.meta["comp_off"][0]),
                         int(e.meta["comp_len"][0]), bo + oo, e.n_out, 0, 0, 0))
            titem.append(ii)
            tchunk.append(0)
    tasks = np.array(recs, dtype=TASK_DTYPE)
    d_tasks = torch.from_numpy(tasks.view(np.uint8).copy()).to(dev)
    n = tasks.size
    plan = Plan(items, tasks, np.array(titem, np.int64), d_tasks, d_in, d_meta, d_out, np.array(out_off),
                np.array(out_len), max_lane)
    plan.extra["task_chunk"] = np.array(tchunk, np.int64)
    plan.d_status = torch.zeros(n, dtype=torch.int32, device=dev)
    plan.d_timing = torch.zeros(2 * n, dtype=torch.int64, device=dev)
    plan.d_counter = torch.zeros(4, dtype=torch.int32, device=dev)
    return plan


def launch(plan: Plan, order=None, dynamic: bool = True, timing: bool = True, blocks_per_sm: int = 0,
           stream=None) -> None:
    """Enqueue gd_batch_decode.  `order` (device int32 tensor or None) is the
    task order: dynamic=True pops it through the work queue, False maps
    order[i] to warp i mod W."""
    import torch
    s = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
    p = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
    rc = lib().gd_batch_decode(p(plan.d_tasks), plan.tasks.size, p(order), 1 if dynamic else 0, plan.max_lane,
                               blocks_per_sm, p(plan.d_counter), p(plan.d_status),
                               p(plan.d_timing) if timing else None, C.c_void_p(s))
    cc.check(rc, "gd_batch_decode")


def n_warps(plan: Plan, blocks_per_sm: int = 0) -> int:
    return int(lib().gd_batch_warps(plan.max_lane, blocks_per_sm))


def verify(plan: Plan, expect: dict | None = None) -> bool:
    """Every task OK and every item's output equal to its raw column, or to
    expect[item index] where given (the reference decoder's output for items
    whose container does not round-trip in the reference itself)."""
    st = plan.d_status.cpu().numpy()
    if (st != 0).any():
        return False
    out = plan.d_out.cpu().numpy()
    for i, (it, o, n) in enumerate(zip(plan.items, plan.out_off, plan.out_len)):
        want = expect[i] if expect and i in expect else it.raw
        if not np.array_equal(out[o:o + n], want):
            return False
    return True


def task_durations_ns(plan: Plan) -> np.ndarray:
    t = plan.d_timing.cpu().numpy().reshape(-1, 2)
    return (t[:, 1] - t[:, 0]).astype(np.float64)


def makespan_ms(plan: Plan, order=None, dynamic=True, reps: int = 3, blocks_per_sm: int = 0) -> float:
    """Median CUDA-event time of the whole batch launch."""
    import torch
    times = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        launch(plan, order, dynamic, timing=False, blocks_per_sm=blocks_per_sm)
        b.record()
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    return float(np.median(times))


# --------------------------------------------------------------------------
# per-task header features (16) for the cost model
# --------------------------------------------------------------------------

N_FEATURES = 16


def header_features(plan: Plan) -> np.ndarray:
    """gd_task_features on the device: (n, 4) float32 -- log2(1 + run
    headers / tokens), literal share (Deflate: first block type / 2), units
    per KiB of output (Deflate: dynamic first block's HLIT + 257 over 286),
    malformed-header flag."""
    import torch
    n = plan.tasks.size
    d = torch.empty(4 * max(n, 1), dtype=torch.float32, device=plan.d_tasks.device)
    s = torch.cuda.current_stream(plan.d_tasks.device).cuda_stream
    cc.check(lib().gd_task_features(C.c_void_p(plan.d_tasks.data_ptr()), n, C.c_void_p(d.data_ptr()),
                                    C.c_void_p(s)), "gd_task_features")
    return d.cpu().numpy().reshape(-1, 4)[:n]


def task_features(plan: Plan) -> np.ndarray:
    """16 features per task, from container metadata and headers only (what
    a scheduler knows before decoding):
      0-4  codec one-hot (brle, RLE v1, RLE v2, LZSS, Deflate)
      5    log2 compressed bytes the task reads (its lane stream for RLE)
      6    log2 output bytes the task writes
      7    compressed / output bytes
      8    lane-stream length skew of the chunk, max / mean (RLE, LZSS)
      9    log2(1 + run headers or tokens)           } the device header
      10   literal share / Deflate first block type   } walk,
      11   log2 chunk (or stream) size                  gd_task_features
      12   units per KiB / Deflate dynamic HLIT share }
      13   malformed-header flag                      }
      14   log2 size of the whole item
      15   constant 1"""
    T = plan.tasks
    n = T.size
    F = np.zeros((n, N_FEATURES), np.float32)
    chunk = plan.extra["task_chunk"]
    item = plan.task_item
    codec = T["codec"].astype(np.int64)
    F[np.arange(n), codec] = 1.0
    src_len = T["src_len"].astype(np.float64)
    dst_len = T["dst_len"].astype(np.float64)
    skew_max = np.ones(n)
    # lane-length statistics of every chunk of the RLE / LZSS items
    lane_items = [i for i, it in enumerate(plan.items) if "col_len" in it.enc.meta]
    if lane_items:
        base = np.zeros(len(plan.items), np.int64)   # first chunk row of each item
        rows, pos = [], 0
        for i in lane_items:
            cl = plan.items[i].enc.meta["col_len"].astype(np.float64).reshape(-1, 32)
            base[i] = pos
            rows.append(cl)
            pos += cl.shape[0]
        L = np.concatenate(rows)                     # (chunks, 32)
        mean = np.maximum(L.mean(1), 1.0)
        sel = np.isin(codec, (1, 2, 3))
        r = base[item[sel]] + chunk[sel]
        skew_max[sel] = (L.max(1) / mean)[r]
        rle = np.isin(codec, (1, 2))
        rr = base[item[rle]] + chunk[rle]
        src_len[rle] = L[rr, T["lane"][rle].astype(np.int64)]
        dst_len[rle] = dst_len[rle] / 32.0
    out_total = np.array([it.enc.n_out for it in plan.items], np.float64)
    H = header_features(plan)
    F[:, 5] = np.log2(src_len + 1.0)
    F[:, 6] = np.log2(dst_len + 1.0)
    F[:, 7] = src_len / np.maximum(dst_len, 1.0)
    F[:, 8] = skew_max
    F[:, 9] = H[:, 0]
    F[:, 10] = H[:, 1]
    cs = T["chunk_size"].astype(np.float64)
    F[:, 11] = np.log2(np.where(cs > 0, cs, T["dst_len"].astype(np.float64)) + 1.0)
    F[:, 12] = np.minimum(H[:, 2], 1024.0) / 64.0
    F[:, 13] = H[:, 3]
    F[:, 14] = np.log2(out_total[item] + 1.0)
    F[:, 15] = 1.0
    return F
