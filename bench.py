#!/usr/bin/env python
"""Decode throughput benchmark (one JSON line on rank 0).

Default (--workload all): every decode configuration on one GPU --
  config 1  RLE v1, 64 MiB int32, 128 KiB chunks, COMP_COL_LEN 128;
  config 2  byte-RLE 256 MiB uint8 (geometric mean-20 runs, 16 Zipf(1.2)
            byte values) + RLE v2 256 MiB int64 (512-value DELTA /
            SHORT_REPEAT / DIRECT / PATCHED_BASE segments), 256 KiB chunks,
            READ_UNIT 32 -- the step `value` is quoted on;
  config 3  LZSS, 1 GiB order-2 Markov + copy bytes, 64 KiB chunks;
  config 4  Deflate/zlib, 1 GiB in 8192 log-uniform chunks, level 6;
  config 5  the mixed-codec batch under five schedules (`mixed`).
Each codec's kernel has its own line in `kernels` (CUDA-event time,
algorithmic bytes, fraction of the measured HBM peak, e2e host call, CPU
baseline).  Synthetic seeded data stands in for the reference's datasets,
which are not available.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload all|brle_rlev2|rlev1|lzss|deflate|mixed|brle_encode|lzss_encode|rlev1_encode|
                               rlev2_encode]
                    [--scale F] [--no-e2e] [--no-cpu] [--no-mixed]

Multi-GPU (torchrun, one process per GPU): every rank decodes its own copy of
the workload (independent chunks, no exchange step), weak scaling, time = max
over ranks.  --impl reference times the reference's CPU decoders on the host
cores (rank 0 only), on inputs built without this library.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

MiB = 1 << 20
GiB = 1 << 30


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# --------------------------------------------------------------------------
# workloads
# --------------------------------------------------------------------------

HEADLINE_METRIC = "decompressed GB/s per codec & % of HBM peak at 1 B200; mixed-batch makespan learned vs static"
HEADLINE = "brle_rlev2"
LABELS = {
    "brle_rlev2": "byte-RLE 256 MiB uint8 + RLE v2 256 MiB int64, 256 KiB chunks, READ_UNIT 32",
    "rlev1": "RLE v1 64 MiB int32, 128 KiB chunks, COMP_COL_LEN 128",
    "lzss": "LZSS 1 GiB Markov+copy bytes, 64 KiB chunks",
    "deflate": "Deflate/zlib 1 GiB in 8192 chunks log-uniform 4 KiB-1 MiB, level 6",
}
DECODE_WORKLOADS = ("rlev1", "brle_rlev2", "lzss", "deflate")
L2_NOTE = "flushed between timed steps (256 MiB write)"


def run_config(workload: str, world: int) -> dict:
    """The `config` of a workload's line; identical in both arms."""
    cfg = {"workload": LABELS.get(workload, workload), "l2": L2_NOTE, "parallelism": f"replicas x{world}"}
    if workload == HEADLINE:
        cfg["columns"] = 2
    return cfg


def deflate_modes(n: int) -> np.ndarray:
    rng = np.random.default_rng(0xD2)
    mode = np.zeros(n, np.uint8)
    r = rng.random(n)
    mode[r < 0.015] = 1
    mode[(r >= 0.015) & (r < 0.03)] = 2
    return mode


def make_workload(name: str, scale: float = 1.0):
    """Returns ([(codec_name, Encoded, raw_bytes_view)], config label)."""
    import compression_b200.codecs as cc
    if name == "brle_rlev2":
        n = int(256 * MiB * scale)
        a = cc.gen_brle_bytes(0xB0, n)
        e1 = cc.brle_encode(a, 256 * 1024)
        v = cc.gen_rlev2_ints(0xB1, n // 8)
        e2 = cc.rlev2_encode(v, 256 * 1024, 32)
        return [("brle", e1, a), ("rlev2", e2, v.view(np.uint8))]
    if name == "rlev1":
        v = cc.gen_rlev1_ints(0xA0, int(64 * MiB * scale) // 4)
        e = cc.rlev1_encode(v, 128 * 1024, 128, 4)
        return [("rlev1", e, v.view(np.uint8))]
    if name == "lzss":
        a = cc.gen_markov_copy(0xC0, int(GiB * scale), 4096)
        e = cc.lzss_encode(a, 64 * 1024)
        return [("lzss", e, a)]
    if name == "deflate":
        total = int(GiB * scale)
        a = cc.gen_markov_copy(0xD0, total, 32768)
        sizes = cc.loguniform_sizes(0xD1, 8192, 4096, MiB, total)
        oo = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
        e = cc.deflate_encode(a, oo, 6, deflate_modes(8192), 1)
        return [("deflate", e, a)]
    raise ValueError(name)


# --------------------------------------------------------------------------
# clocks sampler
# --------------------------------------------------------------------------

class Clocks:
    def __init__(self, gpu_index: int):
        self.samples = []
        self.stop_flag = False
        self.idx = gpu_index
        self.th = None

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        while not self.stop_flag:
            try:
                r = subprocess.run(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={q}", "--format=csv,noheader,nounits"],
                                   capture_output=True, text=True, timeout=5)
                parts = [x.strip() for x in r.stdout.strip().split(",")]
                if len(parts) >= 6:
                    self.samples.append(parts)
            except Exception:
                pass
            time.sleep(0.2)

    def __enter__(self):
        self.th = threading.Thread(target=self._run, daemon=True)
        self.th.start()
        return self

    def __exit__(self, *a):
        self.stop_flag = True
        if self.th:
            self.th.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace('.', '', 1).isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace('.', '', 1).isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[2 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# --------------------------------------------------------------------------
# ranks
# --------------------------------------------------------------------------

def max_over_ranks(values, world: int, device="cpu"):
    """Element-wise maximum of per-rank timings over all ranks (every rank
    gets the result); identity for one rank.  Device tensors for NCCL, CPU
    tensors for gloo."""
    if world <= 1:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def job_rate(bytes_per_rank: int, world: int, ms: float) -> float:
    """Whole-job GB/s: every rank decodes bytes_per_rank (weak scaling) and
    the job takes the slowest rank's time."""
    return bytes_per_rank * world / (ms / 1e3) / 1e9


# --------------------------------------------------------------------------
# CPU baselines (the reference's own CPU decoders, or the oracle port)
# --------------------------------------------------------------------------

REF_BIN = ROOT / "oracle" / "_ref"


class CpuCol:
    """One column prepared for a CPU decoder: a reference harness binary and
    its input file (brle::decode, rlev2::block_decode, lzss::decompress_func,
    compiled from the reference sources into oracle/_ref), or an oracle
    container decoded by the oracle (RLE v1, whose reference decoders are
    GPU-only; Deflate, which the reference decodes on the CPU with zlib)."""

    def __init__(self, name, n_out, exe=None, path=None, cont=None):
        self.name, self.n_out, self.exe, self.path, self.cont = name, int(n_out), exe, path, cont

    @property
    def kind(self) -> str:
        return "reference" if self.exe is not None or self.name == "deflate" else "port"


def _write_lanes(path, lanes, off, per):
    with open(path, "wb") as f:
        f.write(np.array([off.size - 1, per], dtype=np.uint64).tobytes())
        f.write(np.ascontiguousarray(off, dtype=np.uint64).tobytes())
        f.write(lanes.tobytes())
        f.write(bytes(64))


def cpu_cols_from_containers(cols, tmp: Path):
    """CpuCols over this library's containers (byte-identical to the
    reference encoders' output for brle, RLE v2 and LZSS): the lane / column
    streams are exported from the interleaved blocks by the oracle."""
    import oracle
    res = []
    for name, enc, raw in cols:
        path = tmp / f"{name}.bin"
        if name == "brle" and (REF_BIN / "ref_brle").exists():
            ptr = np.ascontiguousarray(enc.meta["ptr"], dtype=np.uint64)
            with open(path, "wb") as f:
                f.write(np.uint32(ptr.size).tobytes())
                f.write(ptr.tobytes())
                f.write(np.uint64(enc.n_out).tobytes())
                f.write(enc.data.tobytes())
            res.append(CpuCol(name, enc.n_out, REF_BIN / "ref_brle", path))
        elif name in ("rlev2", "lzss") and (REF_BIN / f"ref_{name}").exists():
            lanes, off = oracle.export_lanes(enc)
            per = enc.chunk_size // 256 if name == "rlev2" else enc.chunk_size // 32
            _write_lanes(path, lanes, off, per)
            res.append(CpuCol(name, enc.n_out, REF_BIN / f"ref_{name}", path))
        else:
            res.append(CpuCol(name, enc.n_out, cont=_as_container(enc)))
    return res


def _as_container(enc):
    import oracle
    return oracle.Container(enc.codec, enc.data, enc.n_out, enc.n_chunks, enc.chunk_size, dict(enc.meta),
                            {k: v for k, v in enc.params.items() if not k.startswith("_")})


def _zlib_streams(raw: np.ndarray, oo: np.ndarray, modes: np.ndarray, threads: int):
    """Config 4's zlib streams written by Python's zlib (the reference's own
    producer, orig_compressor.py:87), each padded to 8 bytes."""
    import concurrent.futures as cf
    import zlib

    def one(i):
        b = raw[int(oo[i]):int(oo[i + 1])].tobytes()
        if modes[i] == 1:
            co = zlib.compressobj(6, zlib.DEFLATED, 15, 8, zlib.Z_FIXED)
        else:
            co = zlib.compressobj(0 if modes[i] == 2 else 6)
        return co.compress(b) + co.flush()

    with cf.ThreadPoolExecutor(threads) as ex:
        streams = list(ex.map(one, range(oo.size - 1)))
    clen = np.array([len(z) for z in streams], np.uint64)
    padded = (clen + 7) // 8 * 8
    coff = np.concatenate([[0], np.cumsum(padded)]).astype(np.uint64)
    data = np.zeros(int(coff[-1]), np.uint8)
    for z, o in zip(streams, coff[:-1]):
        data[int(o):int(o) + len(z)] = np.frombuffer(z, np.uint8)
    return data, coff, clen


def cpu_cols_reference(workload: str, scale: float, tmp: Path, threads: int):
    """CpuCols of a workload built without this library: the oracle's copy of
    the seeded generators, then the reference's own encoders (brle::encode;
    rlev2::block_encode per lane stream; lzss::compress_func per column, all
    from oracle/_ref), Python's zlib for Deflate, and for RLE v1 -- whose
    only reference encoder is the GPU writer -- the oracle's input builder."""
    import oracle

    def run(*a):
        subprocess.run([str(x) for x in a], check=True, capture_output=True, timeout=900)

    res = []
    if workload == "brle_rlev2":
        n = int(256 * MiB * scale)
        a = oracle.gen_brle_bytes(0xB0, n)
        rawp, cont = tmp / "brle.raw", tmp / "brle.bin"
        a.tofile(rawp)
        run(REF_BIN / "ref_brle", "encode", rawp, cont)
        res.append(CpuCol("brle", n, REF_BIN / "ref_brle", cont))
        v = oracle.gen_rlev2_ints(0xB1, n // 8)
        cs, ru = 256 * 1024, 32
        nc = v.size * 8 // cs
        # lane t of chunk c holds values c*CS/8 + t*RU + k*32*RU + j, j < RU
        lanes = v[:nc * cs // 8].reshape(nc, cs // 8 // (32 * ru), 32, ru).transpose(0, 2, 1, 3)
        vp_ = tmp / "rlev2.raw"
        np.ascontiguousarray(lanes).tofile(vp_)
        run(REF_BIN / "ref_rlev2", "encode_lanes", vp_, cs // 256, threads, tmp / "rlev2.bin")
        res.append(CpuCol("rlev2", v.size * 8, REF_BIN / "ref_rlev2", tmp / "rlev2.bin"))
    elif workload == "rlev1":
        v = oracle.gen_rlev1_ints(0xA0, int(64 * MiB * scale) // 4)
        res.append(CpuCol("rlev1", v.nbytes, cont=oracle.rlev1_encode(v, 128 * 1024, 128, 4)))
    elif workload == "lzss":
        cs = 64 * 1024
        a = oracle.gen_markov_copy(0xC0, int(GiB * scale), 4096)
        nc = a.size // cs
        # column q of a chunk = bytes 4q + 128k .. +3
        cols = a[:nc * cs].reshape(nc, cs // 128, 32, 4).transpose(0, 2, 1, 3)
        cp = tmp / "lzss.raw"
        np.ascontiguousarray(cols).tofile(cp)
        run(REF_BIN / "ref_lzss", "encode_lanes", cp, cs // 32, threads, tmp / "lzss.bin")
        res.append(CpuCol("lzss", nc * cs, REF_BIN / "ref_lzss", tmp / "lzss.bin"))
    elif workload == "deflate":
        total = int(GiB * scale)
        a = oracle.gen_markov_copy(0xD0, total, 32768)
        sizes = oracle.loguniform_sizes(0xD1, 8192, 4096, MiB, total)
        oo = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
        data, coff, clen = _zlib_streams(a, oo, deflate_modes(8192), threads)
        res.append(CpuCol("deflate", total, cont=oracle.Container(
            "deflate", data, total, 8192, 0, {"comp_off": coff, "comp_len": clen, "out_off": oo},
            {"zlib_header": 1})))
    else:
        raise ValueError(workload)
    return res


def cudf_comparator(cont, steps: int, warmup: int):
    """The reference's vendored cuDF inflate (cudf::io::gpuinflate,
    include/cudf_deflate.cuh:1399-1407, compiled for sm_100a into
    oracle/_ref/libref_cudf.so) on config 4's zlib streams, passed as the
    reference's driver passes them (base_deflate.h:66-72: past the 2-byte
    header), in stream order; CUDA events, L2 flushed between launches.
    Returns a dict, or None without a GPU or the library."""
    import ctypes as C
    lib_path = REF_BIN / "libref_cudf.so"
    try:
        import torch
        if not torch.cuda.is_available() or not lib_path.exists():
            return None
    except ImportError:
        return None
    import oracle
    dev = torch.device("cuda", torch.cuda.current_device())
    d_in = torch.from_numpy(np.concatenate([cont.data, np.zeros(64, np.uint8)])).to(dev)
    d_out = torch.zeros(cont.n_out + 64, dtype=torch.uint8, device=dev)
    co, cl, oo = cont.meta["comp_off"], cont.meta["comp_len"], cont.meta["out_off"]
    n = cont.n_chunks
    desc = np.zeros((n, 4), np.uint64)
    desc[:, 0] = d_in.data_ptr() + co[:-1] + 2
    desc[:, 1] = cl - 2
    desc[:, 2] = d_out.data_ptr() + oo[:-1]
    desc[:, 3] = np.diff(oo)
    d_desc = torch.from_numpy(desc.view(np.int64).reshape(-1)).to(dev)
    d_stat = torch.zeros(2 * n, dtype=torch.int64, device=dev)
    L = C.CDLL(str(lib_path))
    s = torch.cuda.current_stream(dev)

    def launch():
        if L.ref_cudf_gpuinflate(C.c_void_p(d_desc.data_ptr()), C.c_void_p(d_stat.data_ptr()), n, 0,
                                 C.c_void_p(s.cuda_stream)) != 0:
            raise RuntimeError("cuDF gpuinflate launch failed")

    launch()
    torch.cuda.synchronize()
    st = d_stat.cpu().numpy().reshape(-1, 2)
    rc, ref = oracle.decode(cont)
    exact = bool(rc == 0 and (st[:, 1] & 0xffffffff == 0).all() and (st[:, 0] == np.diff(oo)).all()
                 and np.array_equal(d_out[:cont.n_out].cpu().numpy(), ref))
    flush = torch.empty(256 * MiB, dtype=torch.uint8, device=dev)
    ts = []
    for k in range(warmup + steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        launch()
        b.record(s)
        torch.cuda.synchronize()
        if k >= warmup:
            ts.append(a.elapsed_time(b))
    ms = statistics.median(ts)
    alg = int(cont.data.nbytes + cont.n_out + 16 * n)
    del d_in, d_out, d_desc, d_stat, flush
    torch.cuda.empty_cache()
    return {"name": "cuDF gpuinflate (the reference's vendored cudf_deflate.cuh, sm_100a)", "ms": round(ms, 4),
            "decomp_gbs": round(cont.n_out / (ms / 1e3) / 1e9, 2), "alg_gbs": round(alg / (ms / 1e3) / 1e9, 2),
            "exact": exact, "order": "stream order, one 128-thread block per stream, as gpuinflate launches"}


def _sub(cont, a, b):
    """Chunks [a, b) of an oracle container as a container of their own."""
    import oracle
    m, cs = cont.meta, cont.chunk_size
    if cont.codec in ("rlev1", "rlev2", "lzss"):
        bo = m["blk_off"]
        meta = {"blk_off": (bo[a:b + 1] - bo[a]).astype(np.uint64), "col_len": m["col_len"][32 * a:32 * b]}
        if "col_map" in m:
            meta["col_map"] = m["col_map"][32 * a:32 * b]
        n_out = min(cont.n_out, b * cs) - a * cs
        return oracle.Container(cont.codec, cont.data[int(bo[a]):int(bo[b])], n_out, b - a, cs, meta,
                                dict(cont.params))
    if cont.codec == "deflate":
        co, cl, oo = m["comp_off"], m["comp_len"], m["out_off"]
        meta = {"comp_off": (co[a:b + 1] - co[a]).astype(np.uint64), "comp_len": cl[a:b],
                "out_off": (oo[a:b + 1] - oo[a]).astype(np.uint64)}
        return oracle.Container("deflate", cont.data[int(co[a]):int(co[b])], int(oo[b] - oo[a]), b - a, 0, meta,
                                dict(cont.params))
    raise ValueError(cont.codec)


def oracle_rate(cont, threads: int, budget_s: float):
    """Decode rate of the oracle over a growing prefix of the container's
    chunks, split over `threads` host threads (ctypes releases the GIL), until
    one pass takes about a quarter of the budget.  Returns (bytes/s, text)."""
    import concurrent.futures as cf
    import oracle
    nch = cont.n_chunks
    take = min(nch, max(threads, 8))
    while True:
        bounds = np.linspace(0, take, threads + 1).astype(int)
        parts = [_sub(cont, int(x), int(y)) for x, y in zip(bounds[:-1], bounds[1:]) if y > x]
        t0 = time.perf_counter()
        with cf.ThreadPoolExecutor(threads) as ex:
            rcs = list(ex.map(lambda e: oracle.decode(e)[0], parts))
        dt = time.perf_counter() - t0
        if any(rcs):
            raise RuntimeError(f"oracle failed on {cont.codec}")
        if dt > budget_s / 4 or take >= nch:
            break
        take = min(nch, take * 4)
    nb = sum(p.n_out for p in parts)
    return nb / dt, f"{take}/{nch} chunks ({nb / MiB:.0f} MiB out)"


def cpu_rates(ccols, threads: int, budget_s: float):
    """Per column: (bytes/s, description, kind) of its CPU decoder on
    `threads` host threads, each for about budget_s / len(ccols) seconds."""
    per = budget_s / max(len(ccols), 1)
    res = []
    for c in ccols:
        if c.exe is not None:
            r = subprocess.run([str(c.exe), "bench", str(c.path), str(threads), str(per)], capture_output=True,
                               text=True, check=True, timeout=120 + 4 * per)
            nb, dt = r.stdout.split()
            rate = int(nb) / float(dt)
            descr = (f"{c.name}: reference {c.exe.name} over the whole column ({c.n_out / MiB:.0f} MiB), "
                     f"repeated {int(nb) // max(c.n_out, 1)}x")
        else:
            rate, d = oracle_rate(c.cont, threads, per)
            descr = ("zlib inflate: " if c.name == "deflate" else "oracle port: ") + d
        res.append((rate, descr, c.kind))
    return res


def combined_rate(ccols, rates):
    """GB/s of decoding all the columns one after the other."""
    t = sum(c.n_out / r for c, (r, _, _) in zip(ccols, rates))
    kinds = {k for _, _, k in rates}
    return sum(c.n_out for c in ccols) / t / 1e9, "; ".join(d for _, d, _ in rates), \
        kinds.pop() if len(kinds) == 1 else "mixed"


# --------------------------------------------------------------------------
# GPU arm
# --------------------------------------------------------------------------

def time_decode(workload, args, world, dev, clk_samples):
    """One decode workload on this GPU: parity of the benchmarked data, then
    `steps` timed steps (CUDA events per kernel on the launching stream, L2
    flushed between steps), the concurrent-stream step for multi-column
    workloads, the e2e host call and the CPU baseline.  Returns a dict."""
    import torch
    import compression_b200.codecs as cc
    t_prep = time.perf_counter()
    cols = make_workload(workload, args.scale)
    t_prep = time.perf_counter() - t_prep
    jobs = [cc.DeviceJob(e, dev) for _, e, _ in cols]
    stream = torch.cuda.current_stream(dev)

    # parity check of the benchmarked data (bit-exact vs the original column)
    for (name, e, raw), j in zip(cols, jobs):
        j.launch()
        torch.cuda.synchronize()
        ok = (j.status() == 0).all() and np.array_equal(j.output(), raw)
        if not ok and (j.status() == 0).all():
            # the reference's own encoder can write a container that does not
            # round-trip (RLE v2 fixed-delta quirk): parity is then checked
            # against the reference decoder (the oracle)
            import oracle
            rc, ref = oracle.decode(e)
            ok = rc == 0 and np.array_equal(j.output(), ref)
        if not ok:
            raise RuntimeError(f"{name}: GPU output differs from the reference decoder")

    flush = torch.empty(256 * MiB, dtype=torch.uint8, device=dev)  # > 126 MB L2

    def step(evs=None):
        for i, j in enumerate(jobs):
            if evs is not None:
                evs[i][0].record(stream)
            j.launch(stream)
            if evs is not None:
                evs[i][1].record(stream)

    for _ in range(args.warmup):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    K = args.steps
    evs = [[[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in jobs] for _ in range(K)]
    torch.cuda.synchronize()
    with Clocks(dev.index or 0) as clk:
        for k in range(K):
            flush.zero_()     # L2 flushed between timed steps, outside the events
            step(evs[k])
        torch.cuda.synchronize()
    clk_samples.extend(clk.samples)
    per_kernel = [[evs[k][i][0].elapsed_time(evs[k][i][1]) for k in range(K)] for i in range(len(jobs))]
    step_ms = [sum(per_kernel[i][k] for i in range(len(jobs))) for k in range(K)]
    serial_ms = statistics.mean(step_ms)
    launches = len(jobs) * K
    conc_ms = None
    if len(jobs) > 1:
        # the step as a reader runs it: the columns are independent, so each
        # decodes on its own stream, all started together; the step is timed
        # on the launching stream from the common start to the last column's end
        side = [torch.cuda.Stream(dev) for _ in jobs]

        def cstep(ev=None):
            start = torch.cuda.Event(enable_timing=ev is not None)
            start.record(stream)
            if ev is not None:
                ev[0] = start
            for sj, j in zip(side, jobs):
                sj.wait_event(start)
                j.launch(sj)
                done = torch.cuda.Event()
                done.record(sj)
                stream.wait_event(done)
            if ev is not None:
                ev[1].record(stream)

        for _ in range(args.warmup):
            flush.zero_()
            cstep()
        torch.cuda.synchronize()
        cev = [[None, torch.cuda.Event(enable_timing=True)] for _ in range(K)]
        with Clocks(dev.index or 0) as clk2:
            for k in range(K):
                flush.zero_()
                cstep(cev[k])
            torch.cuda.synchronize()
        clk_samples.extend(clk2.samples)
        conc_ms = statistics.mean(c[0].elapsed_time(c[1]) for c in cev)
        launches += len(jobs) * K
    ms = max_over_ranks([conc_ms if conc_ms is not None else serial_ms], world, dev)[0]
    out_bytes = sum(e.n_out for _, e, _ in cols)

    # per-kernel roofline: algorithmic bytes = compressed payload + metadata
    # read + decompressed bytes written, per launch, over the kernel's
    # CUDA-event time
    peak, peak_kind = peaks()
    kern = []
    for i, (name, e, _) in enumerate(cols):
        kms = max_over_ranks([statistics.mean(per_kernel[i])], world, dev)[0]
        alg = e.comp_bytes + e.meta_bytes + e.n_out
        gbs = alg / (kms / 1e3) / 1e9
        kern.append({"kernel": name, "workload": LABELS[workload], "ms": round(kms, 4), "alg_bytes": alg,
                     "gbs": round(gbs, 1), "frac": round(gbs / peak, 4), "decomp_gbs": round(e.n_out / (kms / 1e3) / 1e9, 1),
                     "ratio": round(e.comp_bytes / max(e.n_out, 1), 4),
                     "parity": "bit-exact against the input column (the oracle where the reference's encoder "
                               "does not round-trip)"})

    # e2e: the reference-shaped host call (host buffers; H2D + decode + D2H inside)
    e2e = None
    if not args.no_e2e:
        tot_h2d = sum(e.comp_bytes + e.meta_bytes for _, e, _ in cols)
        for _ in range(2):
            for _, e, _ in cols:
                cc.decode_host_pinned(e)
        ts = []
        for _ in range(max(3, min(K, 5))):
            t0 = time.perf_counter()
            for _, e, _ in cols:
                cc.decode_host_pinned(e)
            ts.append(time.perf_counter() - t0)
        e2e_s = max_over_ranks([statistics.median(ts)], world, dev)[0]
        e2e = {"value": round(job_rate(out_bytes, world, e2e_s * 1e3), 3), "unit": "GB/s",
               "h2d_bytes_per_step": int(tot_h2d), "d2h_bytes_per_step": int(out_bytes),
               "path": "gd_*_decompress host C-ABI calls (pinned host buffers)"}
    res = {"workload": workload, "ms": ms, "serial_ms": serial_ms, "conc": conc_ms is not None,
           "value": job_rate(out_bytes, world, ms), "out_bytes": out_bytes, "kernels": kern, "e2e": e2e,
           "launches": launches, "prep_s": t_prep, "cols": cols}
    del jobs, flush
    torch.cuda.empty_cache()
    return res


def attach_cpu(res, threads, budget_s):
    """cpu_baseline of a workload (and of each of its kernels) from the
    reference's own CPU decoders on this library's containers."""
    with tempfile.TemporaryDirectory() as td:
        ccols = cpu_cols_from_containers(res["cols"], Path(td))
        rates = cpu_rates(ccols, threads, budget_s)
    for k, (r, d, kind) in zip(res["kernels"], rates):
        k["cpu_baseline"] = {"value": round(r / 1e9, 3), "unit": "GB/s", "cores": threads, "kind": kind, "sample": d}
    gbs, sample, kind = combined_rate(ccols, rates)
    res["cpu_baseline"] = {"value": round(gbs, 3), "unit": "GB/s", "cores": threads, "kind": kind, "sample": sample}


def run_ours(args, rank, world, local_rank):
    """One decode workload (--workload rlev1 / brle_rlev2 / lzss / deflate)."""
    import torch
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    samples = []
    r = time_decode(args.workload, args, world, dev, samples)
    if rank == 0 and not args.no_cpu:
        attach_cpu(r, os.cpu_count() or 1, 10.0)
    return decode_line(args, world, r, samples)


def decode_line(args, world, r, samples, metric=None):
    peak, peak_kind = peaks()
    dom = max(r["kernels"], key=lambda k: k["ms"])
    traffic = None
    tp = ROOT / "profiles" / "dram_traffic.json"
    if tp.exists() and args.scale == 1.0:
        t = json.loads(tp.read_text()).get(r["workload"], {}).get(dom["kernel"])
        if t:
            traffic = int(t["read"] + t["write"])
    clk = Clocks(0)
    clk.samples = samples
    line = {
        "metric": metric or f"decompressed GB/s ({r['workload']})",
        "value": round(r["value"], 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(r["ms"], 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8/int64" if r["workload"] == HEADLINE else ("u32" if r["workload"] == "rlev1" else "u8"),
        "data": "synthetic (seeded generators)",
        "config": run_config(r["workload"], world),
        "roofline": {"bound": "hbm", "kernel": dom["kernel"], "achieved": dom["gbs"], "peak": peak,
                     "unit": "GB/s", "frac": dom["frac"], "peak_source": peak_kind,
                     "traffic": traffic, "alg_bytes": dom["alg_bytes"],
                     "traffic_source": "profiles/dram_traffic.json (ncu capture of this workload)" if traffic
                     else None},
        "kernels": r["kernels"],
        "gpu_launches": r["launches"],
        "step": f"columns decoded on concurrent streams (one after the other: {r['serial_ms']:.4f} ms)"
        if r["conc"] else "one column",
        "clocks": clk.summary(),
        "e2e": r["e2e"],
    }
    if "cpu_baseline" in r:
        line["cpu_baseline"] = r["cpu_baseline"]
    return line


def run_all(args, rank, world, local_rank):
    """The default run: every decode configuration and the mixed batch.

    `value`, `e2e`, `roofline` and `cpu_baseline` are the byte-RLE + RLE v2
    step (the configuration the metric is quoted on); `kernels` holds every
    codec's kernel (configs 1-4) with its own roofline fraction, e2e and CPU
    baseline; `mixed` holds config 5's makespans (static mapping, FIFO queue,
    size-ordered longest-first, learned longest-first)."""
    import torch
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    threads = os.cpu_count() or 1
    samples = []
    res = {}
    for w in (HEADLINE, "rlev1", "lzss", "deflate"):
        res[w] = time_decode(w, args, world, dev, samples)
        if rank == 0 and not args.no_cpu:
            attach_cpu(res[w], threads, 8.0 if w == HEADLINE else 5.0)
        res[w].pop("cols")
    head = res[HEADLINE]
    line = decode_line(args, world, head, samples, metric=HEADLINE_METRIC)
    kern = []
    for w in ("rlev1", HEADLINE, "lzss", "deflate"):
        for k in res[w]["kernels"]:
            if w != HEADLINE and res[w]["e2e"]:
                k["e2e_gbs"] = res[w]["e2e"]["value"]
            kern.append(k)
    line["kernels"] = kern
    line["gpu_launches"] = sum(r["launches"] for r in res.values())
    if not args.no_mixed:
        m = mixed_run(args, rank, world, local_rank, samples)
        line["mixed"] = m
        line["gpu_launches"] += m.pop("launches")
    clk = Clocks(0)
    clk.samples = samples
    line["clocks"] = clk.summary()
    return line


# --------------------------------------------------------------------------
# mixed-codec batch with the learned scheduler
# --------------------------------------------------------------------------

MIXED_LABEL = ("mixed batch: {n} items log-uniform 4 KiB-2 MiB, {gib:.2f} GiB decompressed, 20/20/10/25/25% "
               "RLE v1/RLE v2/byte-RLE/LZSS/Deflate")


def task_bytes(plan):
    """Bytes each task writes and reads (an RLE lane task writes 1/32 of its
    chunk and reads its own lane stream)."""
    import compression_b200.batch as B
    X = B.task_features(plan)
    return np.exp2(X[:, 6].astype(np.float64)) - 1.0, np.exp2(X[:, 5].astype(np.float64)) - 1.0


def mixed_run(args, rank, world, local_rank, clk_samples):
    """Config 5, the mixed-codec batch: 16384 items (log-uniform 4 KiB - 2 MiB,
    4 GiB decompressed in all; 20% RLE v1, 20% RLE v2, 10% byte-RLE, 25% LZSS,
    25% Deflate) decoded in one persistent launch under eight schedules:

    * static: task i on warp i mod W (the fallback);
    * queue_fifo: the dynamic work queue in task order;
    * size_lpt_out / size_lpt_in: longest-first through the queue with the
      task's decompressed / compressed bytes as its cost (the method without
      the network); size_lpt_out_banded: the same with the codec runs that
      the learned schedule uses;
    * learned_lpt: longest-first by the cost model's prediction (the lane
      tasks of an RLE chunk keyed by their largest prediction, kept
      together; inside bands of a factor of 2, one codec after another), as
      one CUDA-graph replay of [MLP inference -> group maximum -> banded
      order -> batch decode]; learned_order_only is that order computed
      beforehand, learned_per_task every task by its own prediction.

    The cost model is trained on a separate, quarter-size batch of the same
    mix (other seeds), on 200k+ per-task decode times that the batch decoder
    measures itself in random task orders; it is evaluated on this batch."""
    import torch
    import compression_b200.batch as B
    import compression_b200.costmodel as CM

    dev = torch.device("cuda", local_rank)
    n_items = max(64, int(16384 * args.scale))
    total = int(4 * GiB * args.scale)
    t0 = time.perf_counter()
    items = B.make_mixed_batch(0xE0 + rank, n_items, total, 4096, 2 * MiB)
    plan = B.build_plan(items, dev)
    t_build = time.perf_counter() - t0
    n_tasks = plan.tasks.size
    out_bytes = int(plan.out_len.sum())
    comp_bytes = sum(it.enc.comp_bytes + it.enc.meta_bytes for it in items)

    # parity of the benchmarked batch: every item bit-exact against the
    # reference decoder (the oracle); that equals the input column except for
    # containers the reference's own encoder writes wrongly (its RLE v2
    # fixed-delta runs after short repeats), where both decoders agree
    import concurrent.futures as cf
    import oracle
    B.launch(plan, None, dynamic=False, timing=False)
    torch.cuda.synchronize()
    out = plan.d_out.cpu().numpy()
    bad = [i for i, (it, o, n) in enumerate(zip(items, plan.out_off, plan.out_len))
           if not np.array_equal(out[o:o + n], it.raw)]
    expect = {}
    with cf.ThreadPoolExecutor(os.cpu_count() or 1) as ex:
        for i, (rc, ref) in zip(bad, ex.map(lambda i: oracle.decode(items[i].enc), bad)):
            if rc != 0:
                raise RuntimeError(f"mixed batch item {i}: oracle status {rc}")
            expect[i] = ref
    if not B.verify(plan, expect):
        raise RuntimeError("mixed batch: GPU output differs from the reference decoder")
    n_quirk = len(expect)
    del out

    # ---- cost model: trained on a separate batch's self-measured task times ----
    t0 = time.perf_counter()
    titems = B.make_mixed_batch(0xF0 + rank, max(64, n_items // 4), max(total // 4, 64 * MiB), 4096, 2 * MiB)
    tplan = B.build_plan(titems, dev)
    Xt = B.task_features(tplan)
    ys, n_samples, seed = [], 0, 0
    while n_samples < 200_000 or len(ys) < 2:
        ys.append(np.log(np.maximum(CM.measure_tasks(tplan, seed=seed), 1.0)))
        n_samples += tplan.tasks.size
        seed += 1
    model = CM.CostModel(seed=0, device=dev)
    # rows weighted by their measured time: the long tasks, which set the
    # makespan under longest-first placement, are the ones to rank right
    yall = np.concatenate(ys)
    losses = model.train(np.concatenate([Xt] * len(ys)), yall, epochs=8, batch=256, lr=3e-3,
                         weights=np.exp(yall - yall.max()))
    t_train = time.perf_counter() - t0
    del tplan, titems
    X = B.task_features(plan)
    y_eval = np.log(np.maximum(CM.measure_tasks(plan, seed=99), 1.0))
    pred = model.predict(X)
    corr = float(np.corrcoef(pred, y_eval)[0, 1])
    graph = CM.GraphSchedule(plan, model, X)
    out_b, in_b = task_bytes(plan)
    # the learned order itself, computed once, so that the schedule's quality
    # is timed apart from the cost of inference and sorting
    groups, codec = CM.task_groups(plan), plan.tasks["codec"]
    pred32 = model.predict32(X)
    orders = {"size_lpt_out": CM.lpt_order(out_b), "size_lpt_in": CM.lpt_order(in_b),
              "size_lpt_out_banded": CM.lpt_order(np.log(out_b + 1.0), None, codec),
              "learned_order_only": CM.lpt_order(pred32, groups, codec), "learned_per_task": CM.lpt_order(pred)}

    flush = torch.empty(256 * MiB, dtype=torch.uint8, device=dev)
    kinds = ("learned_lpt", "static", "queue_fifo", "size_lpt_out", "size_lpt_in", "size_lpt_out_banded",
             "learned_order_only", "learned_per_task")

    def run(kind):
        if kind == "static":
            B.launch(plan, None, dynamic=False, timing=False)
        elif kind == "queue_fifo":
            B.launch(plan, None, dynamic=True, timing=False)
        elif kind == "learned_lpt":
            graph.replay()
        else:
            B.launch(plan, orders[kind], dynamic=True, timing=False)

    for _ in range(args.warmup):
        for kind in kinds:
            flush.zero_()
            run(kind)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    K = args.steps
    times = {k: [] for k in kinds}
    with Clocks(local_rank) as clk:
        for _ in range(K):
            for kind in kinds:
                flush.zero_()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                run(kind)
                b.record()
                torch.cuda.synchronize()
                times[kind].append(a.elapsed_time(b))
    clk_samples.extend(clk.samples)
    med = dict(zip(kinds, max_over_ranks([statistics.median(times[k]) for k in kinds], world, dev)))
    for kind in kinds:  # every schedule decodes the batch bit-exact
        plan.d_out.zero_()
        run(kind)
        torch.cuda.synchronize()
        if not B.verify(plan, expect):
            raise RuntimeError(f"mixed batch: {kind} schedule output differs")
    ms = med["learned_lpt"]
    peak, peak_kind = peaks()
    ach = (comp_bytes + out_bytes) / (ms / 1e3) / 1e9

    e2e = None
    if not args.no_e2e:
        # through the public batch API with host buffers, two batches in
        # flight: step k's output arena is copied back while step k+1 is
        # copied in and decoded.  A second plan of the same items holds the
        # second set of device arenas; every step copies its inputs in from
        # pinned host memory, replays the learned-schedule graph and copies
        # its whole output back.
        plan2 = B.build_plan(items, dev)
        graph2 = CM.GraphSchedule(plan2, model, X)
        sets = [(plan, graph), (plan2, graph2)]
        h_in = torch.empty(plan.d_in.numel(), dtype=torch.uint8, pin_memory=True)
        h_in.copy_(plan.d_in)
        h_meta = torch.empty(plan.d_meta.numel(), dtype=torch.uint8, pin_memory=True)
        h_meta.copy_(plan.d_meta)
        h_out = [torch.empty(plan.d_out.numel(), dtype=torch.uint8, pin_memory=True) for _ in range(2)]
        s_in, s_run, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
        ev = {k: [torch.cuda.Event(), torch.cuda.Event()] for k in ("inp", "dec", "out")}

        def issue(k):
            j = k % 2
            p, g = sets[j]
            s_in.wait_event(ev["dec"][j])  # the last decode of this set has read its inputs
            with torch.cuda.stream(s_in):
                p.d_in.copy_(h_in, non_blocking=True)
                p.d_meta.copy_(h_meta, non_blocking=True)
            ev["inp"][j].record(s_in)
            s_run.wait_event(ev["inp"][j])
            s_run.wait_event(ev["out"][j])  # the last copy-out of this set has read its output
            with torch.cuda.stream(s_run):
                g.replay()
            ev["dec"][j].record(s_run)
            s_out.wait_event(ev["dec"][j])
            with torch.cuda.stream(s_out):
                h_out[j].copy_(p.d_out, non_blocking=True)
            ev["out"][j].record(s_out)

        for k in range(2):
            issue(k)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        K2 = max(4, min(K, 8))
        t1 = time.perf_counter()
        for k in range(K2):
            issue(2 + k)
        torch.cuda.synchronize()
        e2e_s = max_over_ranks([(time.perf_counter() - t1) / K2], world, dev)[0]
        if not B.verify(plan2, expect) or not torch.equal(h_out[0], h_out[1]):
            raise RuntimeError("mixed batch: pipelined host path output differs")
        e2e = {"value": round(job_rate(out_bytes, world, e2e_s * 1e3), 3), "unit": "GB/s",
               "h2d_bytes_per_step": int(h_in.numel() + h_meta.numel()), "d2h_bytes_per_step": int(h_out[0].numel()),
               "path": "batch API: pinned arenas H2D, graph replay, output arena D2H; two batches in flight "
                       "(copy-out of step k overlaps copy-in and decode of step k+1)",
               "steps": K2}
        del plan2, graph2, h_in, h_meta, h_out

    res = {
        "workload": MIXED_LABEL.format(n=n_items, gib=out_bytes / GiB), "tasks": int(n_tasks),
        "warps": B.n_warps(plan), "value": round(job_rate(out_bytes, world, ms), 2), "unit": "GB/s",
        "makespan_ms": {k: round(v, 3) for k, v in med.items()},
        "learned_gain_vs_static": round(1.0 - ms / med["static"], 4),
        "learned_gain_vs_size_lpt_out": round(1.0 - ms / med["size_lpt_out"], 4),
        "learned_gain_vs_size_lpt_in": round(1.0 - ms / med["size_lpt_in"], 4),
        "learned_order_gain_vs_size_lpt_out": round(1.0 - med["learned_order_only"] / med["size_lpt_out"], 4),
        "learned_gain_vs_size_lpt_out_banded": round(1.0 - ms / med["size_lpt_out_banded"], 4),
        "schedules": {"static": "task i on warp i mod W", "queue_fifo": "work queue, task order",
                      "size_lpt_out": "work queue, longest first by decompressed bytes per task",
                      "size_lpt_in": "work queue, longest first by compressed bytes per task",
                      "size_lpt_out_banded": "size_lpt_out in bands of a factor of 2, one codec after another "
                                             "inside a band",
                      "learned_lpt": "CUDA graph: MLP inference + group maximum + banded sort + work queue (all "
                                     "timed); the 32 lane tasks of an RLE chunk share their largest prediction "
                                     "and stay adjacent; inside bands of a factor of 2 of predicted time, one "
                                     "codec after another",
                      "learned_order_only": "work queue in the learned (grouped, banded) order computed beforehand",
                      "learned_per_task": "work queue, every task by its own prediction (no grouping, no bands)"},
        "cost_model": {"train_batch": "separate quarter-size batch of the same mix (other seeds)",
                       "samples": int(sum(y.size for y in ys)), "epochs": 8, "final_loss": round(float(losses[-1]), 4),
                       "corr_pred_measured_eval_batch": round(corr, 4), "train_s": round(t_train, 1)},
        "roofline": {"bound": "hbm", "kernel": "batch", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(ach / peak, 4), "peak_source": peak_kind, "alg_bytes": int(comp_bytes + out_bytes)},
        "e2e": e2e, "build_s": round(t_build, 1),
        "parity": {"items": len(items), "checked_against": "input column; reference decoder (oracle) for "
                   f"{n_quirk} RLE v2 items its own encoder does not round-trip", "schedules": "all bit-exact"},
        "launches": len(kinds) * K,
    }
    if rank == 0 and not args.no_cpu:
        threads = os.cpu_count() or 1
        gbs, sample = mixed_cpu_sample(items, threads, 6.0)
        res["cpu_baseline"] = {"value": round(gbs, 3), "unit": "GB/s", "cores": threads, "kind": "port",
                               "sample": sample}
    del graph, plan, orders, flush
    torch.cuda.empty_cache()
    return res


def run_mixed(args, rank, world, local_rank):
    """--workload mixed: config 5 alone, as its own line."""
    import torch
    torch.cuda.set_device(torch.device("cuda", local_rank))
    samples = []
    m = mixed_run(args, rank, world, local_rank, samples)
    clk = Clocks(0)
    clk.samples = samples
    line = {"metric": "mixed-batch decompressed GB/s (learned longest-first schedule)", "value": m["value"],
            "unit": "GB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": m["makespan_ms"]["learned_lpt"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8/int32/int64", "data": "synthetic (seeded generators)",
            "config": {"workload": m["workload"], "l2": L2_NOTE, "parallelism": f"replicas x{world}"},
            "gpu_launches": m.pop("launches"), "clocks": clk.summary()}
    line.update({k: v for k, v in m.items() if k not in ("workload", "value", "unit")})
    return line


def mixed_cpu_sample(items, threads: int, budget_s: float):
    """Oracle decode of random items of the mixed batch on the host cores
    (the per-item containers have no single reference CPU entry point)."""
    import concurrent.futures as cf
    import oracle
    rng = np.random.default_rng(1)
    pick = rng.permutation(len(items))
    t1 = time.perf_counter()
    done, nb = 0, 0
    with cf.ThreadPoolExecutor(threads) as ex:
        while time.perf_counter() - t1 < budget_s and done < len(items):
            batch = [items[i].enc for i in pick[done:done + 4 * threads]]
            rcs = list(ex.map(lambda e: oracle.decode(e)[0], batch))
            if any(rcs):
                raise RuntimeError("oracle failed on the mixed batch")
            nb += sum(e.n_out for e in batch)
            done += len(batch)
    dt = time.perf_counter() - t1
    return nb / dt / 1e9, f"{done} random items, {nb / MiB:.0f} MiB out"



# --------------------------------------------------------------------------
# device encoders (RLE v1 / RLE v2 containers written on the GPU)
# --------------------------------------------------------------------------

def encode_column(workload: str, scale: float):
    """The decode workloads' columns: (codec, raw bytes, encoder kwargs, chunk, label)."""
    import compression_b200.codecs as cc
    if workload == "brle_encode":
        a = cc.gen_brle_bytes(0xB0, int(256 * MiB * scale))
        return ("brle", a, {}, 256 * 1024, f"byte-RLE encode of {256 * scale:g} MiB uint8, 256 KiB chunks")
    if workload == "lzss_encode":
        a = cc.gen_markov_copy(0xC0, int(GiB * scale), 4096)
        return ("lzss", a, {}, 64 * 1024, f"LZSS encode of {1024 * scale:g} MiB Markov+copy bytes, 64 KiB chunks")
    if workload == "rlev1_encode":
        v = cc.gen_rlev1_ints(0xA0, int(64 * MiB * scale) // 4)
        return ("rlev1", v.view(np.uint8), dict(comp_col_len=128, elem_bytes=4), 128 * 1024,
                f"RLE v1 encode of {64 * scale:g} MiB int32, 128 KiB chunks, COMP_COL_LEN 128")
    v = cc.gen_rlev2_ints(0xB1, int(256 * MiB * scale) // 8)
    return ("rlev2", v.view(np.uint8), dict(read_unit=32), 256 * 1024,
            f"RLE v2 encode of {256 * scale:g} MiB int64, 256 KiB chunks, READ_UNIT 32")


def host_encode(codec, raw, chunk, kw):
    import compression_b200.codecs as cc
    if codec == "brle":
        return cc.brle_encode(raw, chunk)
    if codec == "lzss":
        return cc.lzss_encode(raw, chunk)
    if codec == "rlev1":
        return cc.rlev1_encode(raw, chunk, kw["comp_col_len"], kw["elem_bytes"])
    return cc.rlev2_encode(raw, chunk, kw["read_unit"])


def host_encode_rate(codec, raw, chunk, kw, budget_s: float):
    """The host encoder (one std::thread per core over chunks) on the whole
    column, repeated for the time budget.  Returns (GB/s of column bytes, reps)."""
    reps, t0 = 0, time.perf_counter()
    while True:
        host_encode(codec, raw, chunk, kw)
        reps += 1
        dt = time.perf_counter() - t0
        if dt >= budget_s:
            return raw.size * reps / dt / 1e9, reps


def run_encode(args, rank, world, local_rank):
    import torch
    import compression_b200.codecs as cc
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    codec, raw, kw, chunk, label = encode_column(args.workload, args.scale)
    host = host_encode(codec, raw, chunk, kw)
    d_col = torch.from_numpy(raw.copy()).to(dev)
    stream = torch.cuda.current_stream(dev)

    # parity: the device container is the host encoder's, and decodes back
    bufs = cc.encode_device(codec, d_col, chunk, **kw)
    torch.cuda.synchronize()
    if codec == "brle":
        size = int(bufs["size"].item())
        nc = host.n_chunks
        ok = np.array_equal(bufs["container"][:size].cpu().numpy(), host.params["container"])
        meta_out = 0  # ptr[] and the sizes are inside the container
    else:
        blk = bufs["blk_off"].cpu().numpy().view(np.uint64)
        size = int(blk[-1])
        nc = blk.size - 1
        meta_out = 8 * (nc + 1) + 8 * 32 * nc
        ok = ((bufs["status"].cpu().numpy() == 0).all() and np.array_equal(blk, host.meta["blk_off"])
              and np.array_equal(bufs["col_len"].cpu().numpy().view(np.uint64), host.meta["col_len"])
              and np.array_equal(bufs["data"][:size].cpu().numpy(), host.data))
        if codec == "lzss":
            meta_out += 32 * nc
            ok = ok and np.array_equal(bufs["col_map"].cpu().numpy(), host.meta["col_map"])
    if not ok:
        raise RuntimeError(f"{codec} device encoder differs from the host encoder")
    job = cc.DeviceJob(host, dev)
    job.launch()
    torch.cuda.synchronize()
    if not ((job.status() == 0).all() and np.array_equal(job.output(), raw)):
        raise RuntimeError(f"{codec} container does not decode back to the column")

    flush = torch.empty(256 * MiB, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        flush.zero_()
        cc.encode_device(codec, d_col, chunk, bufs=bufs, **kw)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    K = args.steps
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    with Clocks(local_rank) as clk:
        for k in range(K):
            flush.zero_()
            evs[k][0].record(stream)
            cc.encode_device(codec, d_col, chunk, bufs=bufs, **kw)
            evs[k][1].record(stream)
        torch.cuda.synchronize()
    ms = max_over_ranks([statistics.mean(a.elapsed_time(b) for a, b in evs)], world, dev)[0]
    value = job_rate(raw.size, world, ms)
    alg = raw.size + size + meta_out  # column in; container (and blk_off, col_len) out
    peak, peak_kind = peaks()
    gbs = alg / (ms / 1e3) / 1e9

    e2e = None
    if not args.no_e2e:
        h_col = torch.from_numpy(raw.copy()).pin_memory()
        d_in = torch.empty_like(d_col)
        if codec == "brle":
            h_data = torch.empty(bufs["container"].numel(), dtype=torch.uint8).pin_memory()
            h_size = torch.empty(1, dtype=torch.int64).pin_memory()

            def host_call():
                d_in.copy_(h_col, non_blocking=True)
                cc.encode_device(codec, d_in, chunk, bufs=bufs)
                h_size.copy_(bufs["size"], non_blocking=True)
                torch.cuda.synchronize()
                n = int(h_size[0])
                h_data[:n].copy_(bufs["container"][:n])
                return n
        else:
            h_data = torch.empty(bufs["data"].numel(), dtype=torch.uint8).pin_memory()
            h_meta = torch.empty(nc + 1 + 32 * nc, dtype=torch.int64).pin_memory()
            h_map = torch.empty(32 * nc, dtype=torch.uint8).pin_memory()

            def host_call():
                d_in.copy_(h_col, non_blocking=True)
                cc.encode_device(codec, d_in, chunk, bufs=bufs, **kw)
                h_meta[:nc + 1].copy_(bufs["blk_off"], non_blocking=True)
                h_meta[nc + 1:].copy_(bufs["col_len"], non_blocking=True)
                if codec == "lzss":
                    h_map.copy_(bufs["col_map"], non_blocking=True)
                torch.cuda.synchronize()
                n = int(h_meta[nc])
                h_data[:n].copy_(bufs["data"][:n])
                return n

        for _ in range(2):
            host_call()
        ts = []
        for _ in range(max(3, min(K, 5))):
            t0 = time.perf_counter()
            host_call()
            ts.append(time.perf_counter() - t0)
        e2e_s = max_over_ranks([statistics.median(ts)], world, dev)[0]
        e2e = {"value": round(job_rate(raw.size, world, e2e_s * 1e3), 3), "unit": "GB/s",
               "h2d_bytes_per_step": int(raw.size), "d2h_bytes_per_step": int(size + meta_out),
               "path": "pinned column H2D, gd_*_encode_device, container D2H"}

    line = {
        "metric": f"encoded GB/s ({codec} device encoder, column bytes in)", "value": round(value, 2),
        "unit": "GB/s", "n_gpus": world, "steps": K, "warmup": args.warmup, "ms_per_step": round(ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {"brle": "u8", "lzss": "u8", "rlev1": "u32"}.get(codec, "int64"), "data": "synthetic (seeded generators)",
        "config": {"workload": label, "l2": "flushed between timed steps (256 MiB write)",
                   "parallelism": f"replicas x{world}", "ratio": round(size / raw.size, 4)},
        "roofline": {"bound": "hbm", "kernel": f"{codec} encode (" + ("regions + header + placement" if codec == "brle" else
                                                                   "columns + ranks + offsets + interleave" if codec == "lzss"
                                                                   else "lane encode + offsets + interleave") + ")",
                     "achieved": round(gbs, 1), "peak": peak, "unit": "GB/s", "frac": round(gbs / peak, 4),
                     "peak_source": peak_kind, "traffic": None, "alg_bytes": alg},
        "gpu_launches": (4 if codec == "lzss" else 3) * K, "step": "one column encoded", "clocks": clk.summary(), "e2e": e2e,
    }
    if rank == 0 and not args.no_cpu:
        threads = os.cpu_count() or 1
        gbs_cpu, reps = host_encode_rate(codec, raw, chunk, kw, 10.0)
        line["cpu_baseline"] = {"value": round(gbs_cpu, 3), "unit": "GB/s", "cores": threads, "kind": "port",
                                "sample": f"host encoder on the whole column, {reps} passes"}
    return line


def run_reference(args, world):
    """The reference's own CPU decoders on all host cores, on inputs built
    without this library (cpu_cols_reference).  `value` is the byte-RLE +
    RLE v2 step (the configuration the metric is quoted on), each step a
    bounded sample: both columns decoded in full, repeated for about 3 s;
    with the default workload, `kernels` adds every other codec's rate."""
    threads = os.cpu_count() or 1
    w = args.workload
    if w == "mixed":
        return {"impl": "reference", "unavailable": "the mixed batch has no single reference CPU entry point; "
                "the default run reports each codec's reference CPU rate"}
    if w.endswith("_encode"):
        codec, raw, kw, chunk, label = encode_column(w, args.scale)
        for _ in range(args.warmup):
            host_encode_rate(codec, raw, chunk, kw, 0.5)
        vals = []
        for _ in range(args.steps):
            gbs, reps = host_encode_rate(codec, raw, chunk, kw, 4.0)
            vals.append(gbs)
        v = statistics.median(vals)
        return {"impl": "reference", "metric": f"encoded GB/s ({codec} device encoder, column bytes in)",
                "value": round(v, 3), "unit": "GB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": None, "higher_is_better": True,
                "config": {"workload": label, "l2": L2_NOTE, "parallelism": f"replicas x{world}",
                           "ratio": None},
                "cpu_baseline": {"value": round(v, 3), "unit": "GB/s", "cores": threads, "kind": "port",
                                 "sample": f"host encoder on the whole column, {reps} passes"},
                "e2e": {"value": round(v, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    head = HEADLINE if w == "all" else w
    kern = []
    with tempfile.TemporaryDirectory() as td:
        tmp = Path(td)
        t0 = time.perf_counter()
        hc = cpu_cols_reference(head, args.scale, tmp, threads)
        prep = time.perf_counter() - t0
        for _ in range(args.warmup):
            cpu_rates(hc, threads, 1.0)
        vals, per_col = [], [[] for _ in hc]
        for _ in range(args.steps):
            rates = cpu_rates(hc, threads, 3.0)
            gbs, sample, kind = combined_rate(hc, rates)
            vals.append(gbs)
            for i, r in enumerate(rates):
                per_col[i].append(r[0])
        for c, rs, r in zip(hc, per_col, rates):
            kern.append({"kernel": c.name, "workload": LABELS[head], "value": round(statistics.median(rs) / 1e9, 3),
                         "unit": "GB/s", "kind": c.kind, "sample": r[1]})
        for f in tmp.iterdir():
            f.unlink()
        if w == "all":
            for ow in ("rlev1", "lzss", "deflate"):
                oc = cpu_cols_reference(ow, args.scale, tmp, threads)
                for c, (r, d, kind) in zip(oc, cpu_rates(oc, threads, 5.0)):
                    kern.append({"kernel": c.name, "workload": LABELS[ow], "value": round(r / 1e9, 3), "unit": "GB/s",
                                 "kind": kind, "sample": d})
                    if c.name == "deflate" and not args.no_gpu_comparator:
                        comp = cudf_comparator(c.cont, 5, 2)
                        if comp is not None:
                            kern[-1]["gpu_comparator"] = comp
                del oc
                for f in tmp.iterdir():
                    f.unlink()
    v = statistics.median(vals)
    return {"impl": "reference", "metric": HEADLINE_METRIC if w == "all" else f"decompressed GB/s ({w})",
            "value": round(v, 3), "unit": "GB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": None, "higher_is_better": True, "config": run_config(head, world),
            "cpu_baseline": {"value": round(v, 3), "unit": "GB/s", "cores": threads, "kind": kind,
                             "sample": sample},
            "e2e": {"value": round(v, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "kernels": kern,
            "inputs": "seeded generators (the oracle's copy), reference encoders (brle::encode, "
                      "rlev2::block_encode, lzss::compress_func), Python zlib; RLE v1 by the oracle's input builder",
            "prep_s": round(prep, 1), "native_libs": native_libs()}


def native_libs():
    """Shared objects of this repository mapped into this process."""
    try:
        with open("/proc/self/maps") as f:
            return sorted({ln.split()[-1].replace(str(ROOT) + "/", "") for ln in f
                           if ln.rstrip().endswith(".so") and str(ROOT) in ln})
    except OSError:
        return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="all", choices=["all", "brle_rlev2", "rlev1", "lzss", "deflate", "mixed",
                                                          "brle_encode", "lzss_encode", "rlev1_encode",
                                                          "rlev2_encode"])
    ap.add_argument("--scale", type=float, default=1.0, help="workload size factor (1.0 = full size)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="default workload without config 5")
    ap.add_argument("--no-gpu-comparator", action="store_true",
                    help="reference arm: skip the reference's cuDF inflate on the GPU")
    ap.add_argument("--tune", action="append", default=[], metavar="CODEC=VALUE",
                    help="pin a decoder knob (autotune.KNOBS), e.g. lzss=512; repeatable")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.tune and args.impl == "ours":
        from compression_b200 import autotune as AT
        for kv in args.tune:
            codec, val = kv.split("=", 1)
            AT.set_knob(AT.KNOBS[codec][0], int(val))

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))

    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args, world)), flush=True)
        return 0

    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    if args.workload == "all":
        line = run_all(args, rank, world, local_rank)
    elif args.workload == "mixed":
        line = run_mixed(args, rank, world, local_rank)
    elif args.workload.endswith("_encode"):
        line = run_encode(args, rank, world, local_rank)
    else:
        line = run_ours(args, rank, world, local_rank)
    if args.tune and isinstance(line, dict) and isinstance(line.get("config"), dict):
        line["config"]["tune"] = args.tune
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
