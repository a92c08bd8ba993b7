#!/usr/bin/env python
"""Decode throughput benchmark (one JSON line on rank 0).

Default workload -- byte-RLE + RLE v2 plain decode: a 256 MiB uint8 column of
runs (geometric mean-20 run length, 16 byte values with Zipf(1.2)
frequencies) in the brle container with 256 KiB chunks, and a 256 MiB int64
column of 512-value segments (DELTA / SHORT_REPEAT / DIRECT / PATCHED_BASE
data) in the RLE v2 transposed container with 256 KiB chunks, READ_UNIT 32.
A step decodes both columns from HBM to HBM.  Synthetic seeded data stands in
for the reference's datasets, which are not available.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload brle_rlev2|rlev1|lzss|deflate|mixed|brle_encode|lzss_encode|rlev1_encode|
                               rlev2_encode]
                    [--scale F]

Multi-GPU (torchrun, one process per GPU): every rank decodes its own copy of
the workload (independent chunks, no exchange step), weak scaling, time = max
over ranks.  --impl reference times the reference's CPU decoders on the host
cores (rank 0 only).
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

def make_workload(name: str, scale: float = 1.0):
    """Returns (label, [(codec_name, Encoded, raw_bytes_view)], config dict)."""
    import compression_b200.codecs as cc
    if name == "brle_rlev2":
        n = int(256 * MiB * scale)
        a = cc.gen_brle_bytes(0xB0, n)
        e1 = cc.brle_encode(a, 256 * 1024)
        v = cc.gen_rlev2_ints(0xB1, n // 8)
        e2 = cc.rlev2_encode(v, 256 * 1024, 32)
        cfg = {"workload": "byte-RLE 256 MiB uint8 + RLE v2 256 MiB int64, 256 KiB chunks, READ_UNIT 32",
               "columns": 2}
        return [("brle", e1, a), ("rlev2", e2, v.view(np.uint8))], cfg
    if name == "rlev1":
        v = cc.gen_rlev1_ints(0xA0, int(64 * MiB * scale) // 4)
        e = cc.rlev1_encode(v, 128 * 1024, 128, 4)
        return [("rlev1", e, v.view(np.uint8))], {"workload": "RLE v1 64 MiB int32, 128 KiB chunks, COMP_COL_LEN 128"}
    if name == "lzss":
        a = cc.gen_markov_copy(0xC0, int(GiB * scale), 4096)
        e = cc.lzss_encode(a, 64 * 1024)
        return [("lzss", e, a)], {"workload": "LZSS 1 GiB Markov+copy bytes, 64 KiB chunks"}
    if name == "deflate":
        total = int(GiB * scale)
        a = cc.gen_markov_copy(0xD0, total, 32768)
        sizes = cc.loguniform_sizes(0xD1, 8192, 4096, MiB, total)
        oo = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
        rng = np.random.default_rng(0xD2)
        mode = np.zeros(8192, np.uint8)
        r = rng.random(8192)
        mode[r < 0.015] = 1
        mode[(r >= 0.015) & (r < 0.03)] = 2
        e = cc.deflate_encode(a, oo, 6, mode, 1)
        return [("deflate", e, a)], {"workload": "Deflate/zlib 1 GiB in 8192 chunks log-uniform 4 KiB-1 MiB, level 6"}
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
# CPU baselines (oracle restatement or the reference's own code)
# --------------------------------------------------------------------------

def cpu_decode_sample(cols, threads: int, budget_s: float = 10.0):
    """Decode a bounded prefix of each column on the host cores with the
    oracle (the checker), in parallel over chunks.  Returns (GB/s of
    decompressed bytes, description)."""
    import concurrent.futures as cf
    import copy
    import oracle
    # one sub-container per chunk range; ctypes releases the GIL
    out_bytes = 0
    t_total = 0.0
    descr = []
    for name, enc, raw in cols:
        nch = enc.n_chunks
        # sample size: start with 8 chunks per thread, grow until ~budget/len(cols)
        take = min(nch, max(threads, 8))
        per = budget_s / len(cols)
        while True:
            parts = _split(enc, take, threads)
            t0 = time.perf_counter()
            with cf.ThreadPoolExecutor(threads) as ex:
                rcs = list(ex.map(lambda e: oracle.decode(e)[0], parts))
            dt = time.perf_counter() - t0
            if any(rcs):
                raise RuntimeError(f"oracle failed on {name}")
            if dt > per / 4 or take >= nch:
                break
            take = min(nch, take * 4)
        nb = sum(p.n_out for p in parts)
        out_bytes += nb
        t_total += dt
        descr.append(f"{name}: {take}/{nch} chunks ({nb / MiB:.0f} MiB out)")
    return out_bytes / t_total / 1e9, "; ".join(descr)


REF_BIN = ROOT / "oracle" / "_ref"


def _ref_container(name, enc, path):
    """Write enc in the file format of the reference harness's bench mode;
    returns the harness binary, or None when the codec has no compiled
    reference CPU decoder."""
    import oracle
    m = enc.meta
    if name == "brle" and (REF_BIN / "ref_brle").exists():
        ptr = np.ascontiguousarray(m["ptr"], dtype=np.uint64)
        with open(path, "wb") as f:
            f.write(np.uint32(ptr.size).tobytes())
            f.write(ptr.tobytes())
            f.write(np.uint64(enc.n_out).tobytes())
            f.write(enc.data.tobytes())
        return REF_BIN / "ref_brle"
    if name in ("rlev2", "lzss") and (REF_BIN / f"ref_{name}").exists():
        lanes, off = oracle.export_lanes(enc)
        per = enc.chunk_size // 256 if name == "rlev2" else enc.chunk_size // 32
        with open(path, "wb") as f:
            f.write(np.array([off.size - 1, per], dtype=np.uint64).tobytes())
            f.write(off.tobytes())
            f.write(lanes.tobytes())
            f.write(bytes(64))
        return REF_BIN / f"ref_{name}"
    return None


def ref_decode_sample(cols, threads: int, budget_s: float = 10.0, prepared=None):
    """Decode rate of the reference's own CPU decoders on the host cores.

    byte-RLE: brle::decode per 256 KiB chunk (brle.h:26-100); RLE v2:
    rlev2::block_decode per lane stream (decoder.h:190); LZSS:
    lzss::decompress_func per column stream (lzss_cpu.h:110) -- compiled from
    the reference sources into oracle/_ref, run on `threads` host threads over
    the whole column, repeated for the time budget.  Codecs without a compiled
    reference decoder (RLE v1, whose decoders are GPU-only; Deflate, which the
    reference decodes on the CPU with zlib) fall back to the oracle, whose
    Deflate path is system zlib.  Returns (GB/s, description, kind,
    prepared) where GB/s is the rate of decoding all columns one after the
    other."""
    prepared = prepared if prepared is not None else {}
    t_total, b_total, descr, kinds = 0.0, 0, [], []
    per = budget_s / len(cols)
    for name, enc, raw in cols:
        if name not in prepared:
            path = Path(tempfile.mkdtemp()) / f"{name}.bin"
            prepared[name] = (_ref_container(name, enc, path), path)
        exe, path = prepared[name]
        if exe is not None:
            r = subprocess.run([str(exe), "bench", str(path), str(threads), str(per)], capture_output=True,
                               text=True, check=True, timeout=120 + 4 * per)
            nb, dt = r.stdout.split()
            rate = int(nb) / float(dt)
            kinds.append("reference")
            descr.append(f"{name}: reference {exe.name} over the whole column ({enc.n_out / MiB:.0f} MiB), "
                         f"repeated {int(nb) // max(enc.n_out, 1)}x")
        else:
            gbs, d = cpu_decode_sample([(name, enc, raw)], threads, budget_s=per)
            rate = gbs * 1e9
            kinds.append("reference" if name == "deflate" else "port")
            descr.append(("zlib inflate: " if name == "deflate" else "oracle port: ") + d)
        t_total += enc.n_out / rate
        b_total += enc.n_out
    kind = kinds[0] if len(set(kinds)) == 1 else "mixed"
    return b_total / t_total / 1e9, "; ".join(descr), kind, prepared


def _split(enc, take, threads):
    """Sub-containers of the first `take` chunks, split into `threads` parts."""
    import compression_b200.codecs as cc
    res = []
    bounds = np.linspace(0, take, threads + 1).astype(int)
    for a, b in zip(bounds[:-1], bounds[1:]):
        if b <= a:
            continue
        res.append(_sub(enc, int(a), int(b)))
    return res


def _sub(enc, a, b):
    import compression_b200.codecs as cc
    m = enc.meta
    cs = enc.chunk_size
    if enc.codec == "brle":
        p = m["ptr"]
        data = enc.data[int(p[a]):int(p[b])]
        ptr = (p[a:b + 1] - p[a]).astype(np.uint64)
        n_out = min(enc.n_out, b * cs) - a * cs
        return cc.Encoded("brle", data, n_out, b - a, cs, {"ptr": ptr})
    if enc.codec in ("rlev1", "rlev2", "lzss"):
        bo = m["blk_off"]
        data = enc.data[int(bo[a]):int(bo[b])]
        meta = {"blk_off": (bo[a:b + 1] - bo[a]).astype(np.uint64), "col_len": m["col_len"][32 * a:32 * b]}
        if "col_map" in m:
            meta["col_map"] = m["col_map"][32 * a:32 * b]
        n_out = min(enc.n_out, b * cs) - a * cs
        return cc.Encoded(enc.codec, data, n_out, b - a, cs, meta, dict(enc.params))
    if enc.codec == "deflate":
        co, cl, oo = m["comp_off"], m["comp_len"], m["out_off"]
        data = enc.data[int(co[a]):int(co[b])]
        meta = {"comp_off": (co[a:b + 1] - co[a]).astype(np.uint64), "comp_len": cl[a:b],
                "out_off": (oo[a:b + 1] - oo[a]).astype(np.uint64)}
        return cc.Encoded("deflate", data, int(oo[b] - oo[a]), b - a, 0, meta, dict(enc.params))
    raise ValueError(enc.codec)


# --------------------------------------------------------------------------
# GPU arm
# --------------------------------------------------------------------------

def run_ours(args, rank, world, local_rank):
    import torch
    import compression_b200.codecs as cc
    import compression_b200 as cb

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    cols, cfg = make_workload(args.workload, args.scale)
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
    with Clocks(local_rank) as clk:
        for k in range(K):
            flush.zero_()     # L2 flushed between timed steps, outside the events
            step(evs[k])
        torch.cuda.synchronize()
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
        with Clocks(local_rank) as clk2:
            for k in range(K):
                flush.zero_()
                cstep(cev[k])
            torch.cuda.synchronize()
        conc_ms = statistics.mean(c[0].elapsed_time(c[1]) for c in cev)
        launches += len(jobs) * K
        if clk2.samples:
            clk.samples.extend(clk2.samples)
    ms = max_over_ranks([conc_ms if conc_ms is not None else serial_ms], world, dev)[0]
    out_bytes = sum(e.n_out for _, e, _ in cols)
    value = job_rate(out_bytes, world, ms)

    # roofline of the dominant kernel: algorithmic bytes = compressed payload
    # + metadata read + decompressed bytes written, per launch
    peak, peak_kind = peaks()
    kern = []
    for i, (name, e, _) in enumerate(cols):
        kms = statistics.mean(per_kernel[i])
        alg = e.comp_bytes + e.meta_bytes + e.n_out
        kern.append({"kernel": name, "ms": round(kms, 4), "alg_bytes": alg,
                     "gbs": round(alg / (kms / 1e3) / 1e9, 1),
                     "decomp_gbs": round(e.n_out / (kms / 1e3) / 1e9, 1),
                     "ratio": round(e.comp_bytes / max(e.n_out, 1), 4)})
    dom = max(kern, key=lambda k: k["ms"])
    traffic = None
    tp = ROOT / "profiles" / "dram_traffic.json"
    if tp.exists() and args.scale == 1.0:
        t = json.loads(tp.read_text()).get(args.workload, {}).get(dom["kernel"])
        if t:
            traffic = int(t["read"] + t["write"])

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

    line = {
        "metric": "decompressed GB/s (byte-RLE + RLE v2 columns)" if args.workload == "brle_rlev2"
        else f"decompressed GB/s ({args.workload})",
        "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": K, "warmup": args.warmup,
        "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8/int64" if args.workload == "brle_rlev2" else "u8", "data": "synthetic (seeded generators)",
        "config": dict(cfg, l2="flushed between timed steps (256 MiB write)", parallelism=f"replicas x{world}"),
        "roofline": {"bound": "hbm", "kernel": dom["kernel"], "achieved": dom["gbs"], "peak": peak,
                     "unit": "GB/s", "frac": round(dom["gbs"] / peak, 4), "peak_source": peak_kind,
                     "traffic": traffic, "alg_bytes": dom["alg_bytes"],
                     "traffic_source": "profiles/dram_traffic.json (ncu capture of this workload)" if traffic
                     else None},
        "kernels": kern,
        "gpu_launches": launches,
        "step": f"columns decoded on concurrent streams (one after the other: {serial_ms:.4f} ms)"
        if conc_ms is not None else "one column",
        "clocks": clk.summary(),
        "e2e": e2e,
    }
    if rank == 0 and not args.no_cpu:
        threads = os.cpu_count() or 1
        gbs, sample, kind, _ = ref_decode_sample(cols, threads)
        line["cpu_baseline"] = {"value": round(gbs, 3), "unit": "GB/s", "cores": threads, "kind": kind,
                                "sample": sample}
    return line


# --------------------------------------------------------------------------
# mixed-codec batch with the learned scheduler
# --------------------------------------------------------------------------

def run_mixed(args, rank, world, local_rank):
    """Mixed-codec batch: 16384 items (log-uniform 4 KiB - 2 MiB, 4 GiB
    decompressed in all; 20% RLE v1, 20% RLE v2, 10% byte-RLE, 25% LZSS, 25%
    Deflate) decoded in one persistent launch.  The cost model is trained on
    the decoder's own per-task timings (random task orders) during warm-up;
    the timed step is the CUDA-graph replay of [MLP inference -> longest-first
    order -> batch decode].  The static mapping (task i -> warp i mod W) and
    the plain FIFO work queue are timed beside it on the same data."""
    import torch
    import compression_b200.batch as B
    import compression_b200.costmodel as CM

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
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

    # ---- training data: self-measured per-task times, random orders ----
    X = B.task_features(plan)
    t0 = time.perf_counter()
    ys, samples = [], 0
    seed = 0
    while samples < 200_000 or len(ys) < 2:
        ys.append(np.log(np.maximum(CM.measure_tasks(plan, seed=seed), 1.0)))
        samples += n_tasks
        seed += 1
    model = CM.CostModel(seed=0, device=dev)
    Xtr = np.concatenate([X] * len(ys))
    ytr = np.concatenate(ys)
    losses = model.train(Xtr, ytr, epochs=8, batch=256, lr=3e-3)
    t_train = time.perf_counter() - t0
    pred = model.predict(X)
    corr = float(np.corrcoef(pred, ys[0])[0, 1])
    graph = CM.GraphSchedule(plan, model, X)

    flush = torch.empty(256 * MiB, dtype=torch.uint8, device=dev)
    fifo = None

    def run(kind):
        if kind == "static":
            B.launch(plan, None, dynamic=False, timing=False)
        elif kind == "queue":
            B.launch(plan, fifo, dynamic=True, timing=False)
        else:
            graph.replay()

    for _ in range(args.warmup):
        for kind in ("static", "queue", "learned"):
            flush.zero_()
            run(kind)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    K = args.steps
    times = {"static": [], "queue": [], "learned": []}
    with Clocks(local_rank) as clk:
        for _ in range(K):
            for kind in ("learned", "static", "queue"):
                flush.zero_()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                run(kind)
                b.record()
                torch.cuda.synchronize()
                times[kind].append(a.elapsed_time(b))
    med = {k: statistics.median(v) for k, v in times.items()}
    ms, med["static"], med["queue"] = max_over_ranks([med["learned"], med["static"], med["queue"]], world, dev)
    plan.d_out.zero_()
    graph.replay()
    torch.cuda.synchronize()
    if not B.verify(plan, expect):
        raise RuntimeError("mixed batch: learned schedule output differs")
    value = job_rate(out_bytes, world, ms)
    peak, peak_kind = peaks()
    alg = comp_bytes + out_bytes
    ach = alg / (ms / 1e3) / 1e9

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
        del plan2, graph2

    line = {
        "metric": "mixed-batch decompressed GB/s (learned longest-first schedule)",
        "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": K, "warmup": args.warmup,
        "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8/int32/int64", "data": "synthetic (seeded generators)",
        "config": {"workload": f"mixed batch: {n_items} items log-uniform 4 KiB-2 MiB, "
                               f"{out_bytes / GiB:.2f} GiB decompressed, 20/20/10/25/25% "
                               "RLE v1/RLE v2/byte-RLE/LZSS/Deflate", "tasks": int(n_tasks),
                   "warps": B.n_warps(plan), "l2": "flushed between timed launches (256 MiB write)",
                   "parallelism": f"replicas x{world}"},
        "makespan_ms": {"static": round(med["static"], 3), "queue_fifo": round(med["queue"], 3),
                        "learned_lpt": round(ms, 3)},
        "learned_gain_vs_static": round(1.0 - ms / med["static"], 4),
        "cost_model": {"samples": int(len(ytr)), "epochs": 8, "final_loss": round(float(losses[-1]), 4),
                       "corr_pred_measured": round(corr, 4), "train_s": round(t_train, 1)},
        "roofline": {"bound": "hbm", "kernel": "batch", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(ach / peak, 4), "peak_source": peak_kind, "traffic": None},
        "gpu_launches": 2 * K,
        "clocks": clk.summary(),
        "e2e": e2e,
        "build_s": round(t_build, 1),
        "parity": {"items": len(items), "checked_against": "input column; reference decoder (oracle) for "
                   f"{n_quirk} RLE v2 items its own encoder does not round-trip"},
    }
    if rank == 0 and not args.no_cpu:
        threads = os.cpu_count() or 1
        gbs, sample = mixed_cpu_sample(items, threads, 10.0)
        line["cpu_baseline"] = {"value": round(gbs, 3), "unit": "GB/s", "cores": threads, "kind": "port",
                                "sample": sample}
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


def run_reference(args):
    """The reference's own CPU decoders (oracle/_ref, compiled from the
    reference sources) on all host cores; the oracle port for codecs whose
    reference decoders are GPU-only."""
    threads = os.cpu_count() or 1
    vals, prep = [], None
    if args.workload == "mixed":
        import compression_b200.batch as B
        n_items = max(64, int(16384 * args.scale))
        items = B.make_mixed_batch(0xE0, n_items, int(4 * GiB * args.scale), 4096, 2 * MiB)
        cfg = {"workload": f"mixed-codec batch, {n_items} items, {4 * args.scale:g} GiB decompressed"}
        for _ in range(args.warmup):
            mixed_cpu_sample(items, threads, 1.0)
        for _ in range(args.steps):
            gbs, sample = mixed_cpu_sample(items, threads, 4.0)
            vals.append(gbs)
        kind = "port"
    elif args.workload.endswith("_encode"):
        codec, raw, kw, chunk, label = encode_column(args.workload, args.scale)
        cfg = {"workload": label}
        for _ in range(args.warmup):
            host_encode_rate(codec, raw, chunk, kw, 0.5)
        for _ in range(args.steps):
            gbs, reps = host_encode_rate(codec, raw, chunk, kw, 4.0)
            vals.append(gbs)
            sample = f"host encoder on the whole column, {reps} passes"
        kind = "port"
    else:
        cols, cfg = make_workload(args.workload, args.scale)
        for _ in range(args.warmup):
            _, _, _, prep = ref_decode_sample(cols, threads, budget_s=1.0, prepared=prep)
        for _ in range(args.steps):
            gbs, sample, kind, prep = ref_decode_sample(cols, threads, budget_s=4.0, prepared=prep)
            vals.append(gbs)
    v = statistics.median(vals)
    metric = ("decompressed GB/s (byte-RLE + RLE v2 columns)" if args.workload == "brle_rlev2"
              else f"encoded GB/s ({args.workload.split('_')[0]} device encoder, column bytes in)"
              if args.workload.endswith("_encode") else f"decompressed GB/s ({args.workload})")
    return {"impl": "reference", "metric": metric,
            "value": round(v, 3), "unit": "GB/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": None, "higher_is_better": True, "config": cfg,
            "cpu_baseline": {"value": round(v, 3), "unit": "GB/s", "cores": threads, "kind": kind,
                             "sample": sample},
            "e2e": {"value": round(v, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="brle_rlev2", choices=["brle_rlev2", "rlev1", "lzss", "deflate", "mixed",
                                                                 "brle_encode", "lzss_encode", "rlev1_encode",
                                                                 "rlev2_encode"])
    ap.add_argument("--scale", type=float, default=1.0, help="workload size factor (1.0 = full size)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))

    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return 0

    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    if args.workload == "mixed":
        line = run_mixed(args, rank, world, local_rank)
    elif args.workload.endswith("_encode"):
        line = run_encode(args, rank, world, local_rank)
    else:
        line = run_ours(args, rank, world, local_rank)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
