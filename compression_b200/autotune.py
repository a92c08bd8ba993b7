"""Autotuner for the decoders' launch shapes and kernel variants.

Every knob of include/gd.h (gd_tune_key) selects among kernel variants that
are compiled into libgd.so or sets a launch shape:

  inflate  GD_TUNE_INFLATE_VARIANT        1, 2: one warp per stream, no window, 2 / 4 per block
                                          3: one warp per stream with a 32 KiB window
                                          4, 5: decoder + writer pair, no window, 2 / 4 per block
                                          6: decoder + writer pair with the window
                                          7-13: pairs with a 16 / 8 / 4 KiB window, smaller buffers
                                          0: 12 for >= 4 streams per SM, else 6
  brle     GD_TUNE_BRLE_BLOCKS_PER_SM     grid = value x SMs
  rlev1    GD_TUNE_RLEV1_LANES_PER_BLOCK  lane streams (warps) per block
  rlev2    GD_TUNE_RLEV2_LANES_PER_BLOCK  lane streams (warps) per block
  lzss     GD_TUNE_LZSS_WARPS_PER_BLOCK   0: a warp per chunk, a lane per column, output in rounds
                                          (1 chunk per block), 4: the same, 4 per block; 512 / 256:
                                          16 / 8 lanes per column, 1: a lane per column (these stage
                                          the whole chunk in shared memory)

For the batched decoder the tuned quantity is its blocks per SM (4 warps each),
which sets how many tasks run at once against how much shared memory each
gets.

The tuner times each candidate on the caller's own (device-resident) input
with CUDA events, flushing L2 between repetitions, checks that every candidate
decodes bit-identically to the first, keeps the fastest, and leaves it set.
Results can be kept in a JSON file keyed by device name, codec and input size
(log2 bucket), so later processes apply them without re-measuring.
"""
from __future__ import annotations

import json
import math
import os
import statistics
from pathlib import Path

import numpy as np

from . import codecs as cc
from ._lib import lib

TUNE_INFLATE_VARIANT = 0
TUNE_BRLE_BLOCKS_PER_SM = 1
TUNE_RLEV1_LANES_PER_BLOCK = 2
TUNE_RLEV2_LANES_PER_BLOCK = 3
TUNE_LZSS_WARPS_PER_BLOCK = 4

# codec -> (knob, candidate values; the first is the built-in default)
KNOBS = {
    "deflate": (TUNE_INFLATE_VARIANT, [0, 6, 12, 10, 4]),
    "brle": (TUNE_BRLE_BLOCKS_PER_SM, [8, 4, 16]),
    "rlev1": (TUNE_RLEV1_LANES_PER_BLOCK, [8, 4]),
    "rlev2": (TUNE_RLEV2_LANES_PER_BLOCK, [8, 4]),
    "lzss": (TUNE_LZSS_WARPS_PER_BLOCK, [0, 4, 512, 256]),
}


def set_knob(key: int, value: int) -> int:
    prev = lib().gd_tune_set(key, value)
    if prev < 0:
        raise ValueError(f"bad tuning knob {key}={value}")
    return prev


def get_knob(key: int) -> int:
    return int(lib().gd_tune_get(key))


def _time_ms(fn, reps: int, flush) -> float:
    import torch
    ts = []
    for _ in range(reps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    return statistics.median(ts)


def _flush_buffer(device):
    import torch
    return torch.empty(256 << 20, dtype=torch.uint8, device=device)  # > 126 MB L2


def size_bucket(nbytes: int) -> int:
    return int(math.log2(max(nbytes, 1)))


class Tuner:
    """Measures knob candidates and remembers the winners."""

    def __init__(self, cache_path: str | os.PathLike | None = None, device="cuda"):
        import torch
        self.torch = torch
        self.device = torch.device(device)
        self.name = torch.cuda.get_device_name(self.device)
        self.cache_path = Path(cache_path) if cache_path else None
        self.results: dict = {}
        if self.cache_path and self.cache_path.exists():
            self.results = json.loads(self.cache_path.read_text())

    def key(self, codec: str, nbytes: int) -> str:
        return f"{self.name}|{codec}|{size_bucket(nbytes)}"

    def apply(self, codec: str, nbytes: int) -> bool:
        """Set the remembered knob for this codec and size; False if none."""
        r = self.results.get(self.key(codec, nbytes))
        if r is None or codec not in KNOBS:
            return False
        set_knob(KNOBS[codec][0], int(r["value"]))
        return True

    def save(self) -> None:
        if self.cache_path:
            self.cache_path.write_text(json.dumps(self.results, indent=1, sort_keys=True))

    def tune_job(self, job: "cc.DeviceJob", reps: int = 5) -> dict:
        """Tune the knob of job's codec on job's own input; leaves the best set."""
        codec = job.enc.codec
        if codec not in KNOBS:
            return {}
        knob, values = KNOBS[codec]
        flush = _flush_buffer(self.device)
        times, ref = {}, None
        for v in values:
            set_knob(knob, v)
            job.launch()  # warm-up (first launch sets kernel attributes)
            self.torch.cuda.synchronize()
            st = job.status()
            if (st != 0).any():
                raise RuntimeError(f"{codec}: candidate {v} failed with status {np.unique(st)}")
            out = job.output()
            if ref is None:
                ref = out.copy()
            elif not np.array_equal(out, ref):
                raise RuntimeError(f"{codec}: candidate {v} decodes differently")
            times[v] = _time_ms(job.launch, reps, flush)
        best = min(times, key=times.get)
        set_knob(knob, best)
        res = {"codec": codec, "knob": knob, "value": int(best), "ms": {str(k): round(t, 4) for k, t in times.items()}}
        self.results[self.key(codec, job.enc.n_out)] = res
        return res

    def tune_batch(self, plan, order=None, candidates=None, reps: int = 3) -> dict:
        """Blocks per SM of the persistent batch decoder (dynamic queue)."""
        from . import batch as B
        flush = _flush_buffer(self.device)
        if candidates is None:
            candidates = [0, 1, 2, 3, 4]
        times = {}
        for bps in candidates:
            B.launch(plan, order, dynamic=True, timing=False, blocks_per_sm=bps)
            self.torch.cuda.synchronize()
            times[bps] = _time_ms(lambda: B.launch(plan, order, dynamic=True, timing=False, blocks_per_sm=bps),
                                  reps, flush)
        best = min(times, key=times.get)
        res = {"codec": "batch", "blocks_per_sm": int(best), "ms": {str(k): round(t, 4) for k, t in times.items()}}
        self.results[self.key("batch", int(plan.out_len.sum()))] = res
        return res
