"""Regenerate the golden fixtures from the reference's own codecs.

    python oracle/build.py --ref          # builds oracle/_ref/ref_* from the reference sources
    python tests/golden/make_golden.py    # writes tests/golden/*.npz

Inputs come from the seeded generators (compression_b200.codecs) and a few
hand-picked patterns.  For each input the reference's own encoder output and
the reference's own decoder output are stored, so the tests can check (a) the
library's encoders reproduce the reference bytes exactly and (b) the oracle
and the GPU decoders recover the input from the reference's streams.
Deflate fixtures come from Python's zlib, the producer the reference's
container is written with (orig_compressor.py:87).  The RLE v1 and byte-RLE
flag containers have GPU-only codecs in the reference: their writers and
readers run on host threads (oracle/ref/host_cuda.h), compiled from the
reference's own kernels.
"""
from __future__ import annotations

import subprocess
import sys
import tempfile
import zlib
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
import compression_b200.codecs as cc  # noqa: E402

REF = ROOT / "oracle" / "_ref"
OUT = Path(__file__).resolve().parent


def run(*args):
    subprocess.run([str(a) for a in args], check=True, stdout=subprocess.DEVNULL)


def negative_constant_run(tmp: Path):
    """An RLE v2 lane the reference's own encoder writes as a corrupt stream:
    128 equal negative values reach determineEncoding through the fixed-run
    path (var_runlen 0), is_safe_subtract's `smaller - INT64_MIN` wraps and
    calls the run unsafe, and write_direct stores var_runlen - 1 = 0xffff as
    the length field (a DIRECT run claiming 512 values).  Only the encoder
    output is stored: the reference decoder would read past its run.  The
    lane is lane 0 of the last chunk of a 70000-value constant -5 column in
    256 KiB chunks, READ_UNIT 32 (160 values, then the zero padding)."""
    lane = np.concatenate([np.full(160, -5, np.int64), np.zeros(864, np.int64)])
    lane.tofile(tmp / "v")
    run(REF / "ref_rlev2", "encode", tmp / "v", tmp / "vs")
    np.savez_compressed(OUT / "rlev2_negconst.npz", raw=lane, enc=np.fromfile(tmp / "vs", np.uint8))


def _interleaved(prefix: Path, with_map: bool):
    out = {"data": np.fromfile(f"{prefix}.data", np.uint8), "col_len": np.fromfile(f"{prefix}.col_len", np.uint64),
           "blk_off": np.fromfile(f"{prefix}.blk_off", np.uint64)}
    if with_map:
        out["col_map"] = np.fromfile(f"{prefix}.col_map", np.uint8)
    return out


def gpu_only_codecs(tmp: Path, rng):
    """RLE v1 (rle_v1::compress_gpu / decompress_gpu: setup_deflate,
    reduction_scan, deflate; inflate) and the byte-RLE flag containers
    (brle_trans::compress_gpu / decompress_gpu, brle_gpu_4B.h's
    compress_gpu / decompress_gpu): the reference writer's container and the
    reference reader's output for each input."""
    # ---- RLE v1: (values, element bytes, chunk size, COMP_COL_LEN) ----
    lit_edges = np.concatenate([np.arange(127, dtype=np.int64) * 1000, np.full(5, 7), np.arange(128) * 999,
                                np.arange(130) * 2 + 5, np.arange(131) * 3, [0xFFFFFFFF, 0, 0xFFFFFFFF]])
    cases = [
        (cc.gen_rlev1_ints(0xA0, 4 * 32768), 4, 128 * 1024, 128),                       # config 1's data
        (cc.gen_rlev1_ints(0xA1, 7 * 2048 + 100), 4, 8192, 8),                          # partial last chunk
        (cc.gen_rlev2_ints(0xA2, 5 * 2048 + 3), 8, 16384, 64),                          # 8-byte values
        (np.resize(lit_edges, 4 * 8192).astype(np.uint32), 4, 32768, 256),            # group / run limits
        (np.resize(np.repeat(rng.integers(0, 1 << 20, 600), rng.integers(1, 140, 600)),
                   2 * 8192).astype(np.uint32), 4, 8192, 16),                            # constant runs
        ((np.arange(4096, dtype=np.int64) * -5 + 1000).astype(np.uint32), 4, 16384, 32),  # negative deltas
    ]
    rz = {}
    for i, (vals, eb, chunk, ccl) in enumerate(cases):
        raw = np.ascontiguousarray(vals).view(np.uint8)
        raw.tofile(tmp / "r1")
        run(REF / "ref_rlev1_host", "encode", tmp / "r1", eb, chunk, ccl, tmp / "r1o")
        run(REF / "ref_rlev1_host", "decode", tmp / "r1o", eb, chunk, ccl, raw.size, tmp / "r1d")
        rz[f"raw{i}"] = raw
        for k, v in _interleaved(tmp / "r1o", False).items():
            rz[f"{k}{i}"] = v
        rz[f"dec{i}"] = np.fromfile(tmp / "r1d", np.uint8)
        rz[f"params{i}"] = np.array([eb, chunk, ccl], np.uint64)
    np.savez_compressed(OUT / "rlev1_golden.npz", **rz)

    # ---- byte-RLE flag containers: 1-byte symbols (4 KiB chunks, an even
    # count: the reference reader decodes chunks in pairs) and 4-byte symbols
    # (8 KiB chunks) ----
    for name, exe, chunk, cases in [
        ("brle_trans", "ref_brle_trans_host", 4096, [
            cc.gen_brle_bytes(7, 4096 * 40), np.zeros(4096 * 2, np.uint8), rng.integers(0, 256, 4096 * 4).astype(np.uint8),
            np.repeat(rng.integers(0, 4, 3000), rng.integers(1, 12, 3000)).astype(np.uint8)[:4096 * 6],
            np.resize(np.array([1, 2, 3, 4, 5, 6, 7] + [9] * 121, np.uint8).repeat(1), 4096 * 2)]),
        ("brle_trans4", "ref_brle_trans4_host", 8192, [
            np.resize(np.repeat(rng.integers(0, 6, 20000), rng.integers(1, 20, 20000)).astype(np.uint32),
                      8192 * 10 // 4).view(np.uint8).copy(),
            np.zeros(8192 * 2, np.uint8), rng.integers(0, 256, 8192 * 3).astype(np.uint8),
            cc.gen_rlev1_ints(3, 8192 * 4 // 4).view(np.uint8).copy()])]:
        bz = {}
        for i, raw in enumerate(cases):
            raw = np.ascontiguousarray(raw[:raw.size // chunk * chunk])
            raw.tofile(tmp / "b")
            run(REF / exe, "encode", tmp / "b", tmp / "bo")
            run(REF / exe, "decode", tmp / "bo", raw.size, tmp / "bd")
            bz[f"raw{i}"] = raw
            for k, v in _interleaved(tmp / "bo", True).items():
                bz[f"{k}{i}"] = v
            bz[f"dec{i}"] = np.fromfile(tmp / "bd", np.uint8)
        np.savez_compressed(OUT / f"{name}_golden.npz", **bz)


def main():
    tmp = Path(tempfile.mkdtemp())
    rng = np.random.default_rng(20261203)

    # ---- byte-RLE containers (brle.h) ----
    cases = [cc.gen_brle_bytes(1, 3 * 262144 + 777), cc.gen_brle_bytes(2, 100),
             np.zeros(5000, np.uint8), np.arange(70000, dtype=np.uint8),
             rng.integers(0, 3, 300000).astype(np.uint8),
             np.repeat(rng.integers(0, 256, 2000), rng.integers(1, 300, 2000)).astype(np.uint8)]
    bz = {}
    for i, raw in enumerate(cases):
        raw.tofile(tmp / "in")
        run(REF / "ref_brle", "encode", tmp / "in", tmp / "enc")
        run(REF / "ref_brle", "decode", tmp / "enc", tmp / "dec")
        bz[f"raw{i}"] = raw
        bz[f"enc{i}"] = np.fromfile(tmp / "enc", np.uint8)
        bz[f"dec{i}"] = np.fromfile(tmp / "dec", np.uint8)
    np.savez_compressed(OUT / "brle_golden.npz", **bz)

    # ---- LZSS column streams (lzss_cpu.h compress_func / decompress_func) ----
    lz = {}
    big = cc.gen_markov_copy(3, 64 * 1024, 4096)
    cols = []
    for q in (0, 7, 31):  # the 2 KiB columns of a 64 KiB chunk, as the container stripes them
        cols.append(np.concatenate([big[128 * k + 4 * q: 128 * k + 4 * q + 4] for k in range(512)]))
    cols += [cc.gen_markov_copy(4, 4096, 4096), np.zeros(2048, np.uint8),
             np.tile(np.arange(7, dtype=np.uint8), 300)[:2048], rng.integers(0, 256, 1024).astype(np.uint8)]
    for i, col in enumerate(cols):
        col.tofile(tmp / "c")
        run(REF / "ref_lzss", "encode", tmp / "c", tmp / "cs")
        run(REF / "ref_lzss", "decode", tmp / "cs", col.size, tmp / "cd")
        lz[f"raw{i}"] = col
        lz[f"enc{i}"] = np.fromfile(tmp / "cs", np.uint8)
        lz[f"dec{i}"] = np.fromfile(tmp / "cd", np.uint8)
    np.savez_compressed(OUT / "lzss_golden.npz", **lz)

    # ---- RLE v2 lane streams (encoder.h block_encode / decoder.h block_decode) ----
    rv = {}
    v = cc.gen_rlev2_ints(5, 32 * 1024)
    lanes = [v[t * 32 + np.concatenate([np.arange(k * 1024, k * 1024 + 32) for k in range(32)])] for t in (0, 5, 31)]
    lanes += [np.arange(1024, dtype=np.int64) * 3 + 11, np.full(700, 42, np.int64),
              rng.integers(0, 2 ** 12, 1024).astype(np.int64) + (rng.random(1024) < 0.02) * (1 << 40),
              np.cumsum(rng.integers(1, 1000, 1024)).astype(np.int64) + 1600000000000,
              rng.integers(0, 2 ** 17, 1024).astype(np.int64)]
    for i, lane in enumerate(lanes):
        lane = lane.astype(np.int64)
        lane.tofile(tmp / "v")
        run(REF / "ref_rlev2", "encode", tmp / "v", tmp / "vs")
        run(REF / "ref_rlev2", "decode", tmp / "vs", lane.size, tmp / "vd")
        rv[f"raw{i}"] = lane
        rv[f"enc{i}"] = np.fromfile(tmp / "vs", np.uint8)
        rv[f"dec{i}"] = np.fromfile(tmp / "vd", np.int64)
    np.savez_compressed(OUT / "rlev2_golden.npz", **rv)

    # ---- an RLE v2 lane the reference's own encoder writes wrongly: a
    # 12-value constant run after two short repeats becomes a fixed-delta run
    # with a non-zero delta (lane 20 of a 5120-value generator column) ----
    col = cc.gen_rlev2_ints(0xE0 * 100003 + 9149, 5120)
    lane = col[20 * 32 + np.concatenate([np.arange(k * 1024, k * 1024 + 32) for k in range(5)])].astype(np.int64)
    lane.tofile(tmp / "v")
    run(REF / "ref_rlev2", "encode", tmp / "v", tmp / "vs")
    run(REF / "ref_rlev2", "decode", tmp / "vs", lane.size, tmp / "vd")
    np.savez_compressed(OUT / "rlev2_quirk.npz", raw=lane, enc=np.fromfile(tmp / "vs", np.uint8),
                        dec=np.fromfile(tmp / "vd", np.int64))

    negative_constant_run(tmp)

    gpu_only_codecs(tmp, rng)

    # ---- Deflate chunks (Python zlib, level 6 / 9 as orig_compressor.py) ----
    dz = {}
    raw = cc.gen_markov_copy(6, 300000, 32768)
    for i, (a, b, lvl) in enumerate([(0, 4096, 6), (4096, 150000, 6), (150000, 300000, 9), (0, 1000, 0)]):
        dz[f"raw{i}"] = raw[a:b]
        dz[f"enc{i}"] = np.frombuffer(zlib.compress(raw[a:b].tobytes(), lvl), np.uint8)
        dz[f"lvl{i}"] = np.array([lvl])
    np.savez_compressed(OUT / "deflate_golden.npz", **dz)
    print("fixtures written to", OUT)


if __name__ == "__main__":
    main()
