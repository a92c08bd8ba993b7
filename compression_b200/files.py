"""The reference's on-disk layouts for the compressed containers.

Each writer produces the files the reference's own compressors write, and
each reader returns the Encoded container the decoders take, so a column
compressed by the reference's tools can be decoded here and the other way
round.  Layouts (ZaidQureshi/compression):

  byte-RLE          one file: [u32 n_ptr][u64 ptr[n_ptr]][u64 total][data]
                    (include/brle/brle.h:278-303)
  LZSS              <path>: the interleaved blocks; <path>.meta: the metadata
                    sidecar [u64 num][u64 lens[num]][blob]... with the blobs
                    chunk_size (u64), blk_offset (u64 x n+1), col_len
                    (u64 x 32n, sorted), col_map (u8 x 32n)
                    (include/utils.h:46-119, include/lzss/lzss_gpu2.h:2090-2108)
  RLE v1            <path>: [u64 in_n_bytes][blocks]; side files
                    <dir>/rle_v1_col_len.bin (u64 x 32n) and
                    rle_v1_blk_offset.bin (u64 x n+1) (include/rle_v1/rlev1.h:70-87)
  flag byte-RLE     <path>: the blocks; side files <dir>/col_len.bin,
  (1- and 4-byte    col_map.bin, blk_offset.bin (include/brle/brle_trans.h:646-657,
  symbols)          include/brle/brle_gpu_4B.h:700-711)
  Deflate           <id>_comp.bin: zlib streams each zero-padded to 8 bytes;
                    <id>_col_len.bin: u64 padded lengths; <id>_blk_offset.bin:
                    [u64 total][u64 0][u64 cumulative padded offsets]
                    (orig_compressor.py:44-126); uniform chunks, the last one
                    zero-padded before compressing
  cuDF single file  [u64 chunk_size][u64 n_chunks][u64 stream_len[n]][zlib
                    streams, unpadded] (rapids_compressor.py:222-280, read by
                    base_deflate.h:42-73)

The readers and writers are host I/O (numpy; the cuDF writer compresses with
zlib as the reference's producer does); decoding goes through
codecs.DeviceJob / decode_host, and decode_cudf_single runs the cuDF
reader's flow on gd_gpuinflate.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

from .codecs import Encoded


def _u64(x) -> bytes:
    return np.asarray(x, dtype=np.uint64).tobytes()


def _read_u64(path, count=-1, offset=0) -> np.ndarray:
    return np.fromfile(path, dtype=np.uint64, count=count, offset=offset)


# ---------------------------------------------------------------------------
# byte-RLE: the container is the file
# ---------------------------------------------------------------------------

def write_brle(enc: Encoded, path) -> None:
    Path(path).write_bytes(enc.params["container"].tobytes())


def read_brle(path) -> Encoded:
    cont = np.fromfile(path, dtype=np.uint8)
    n_ptr = int(cont[:4].view(np.uint32)[0])
    ptr = cont[4:4 + 8 * n_ptr].copy().view(np.uint64)
    hdr = 4 + 8 * n_ptr
    total = int(cont[hdr:hdr + 8].view(np.uint64)[0])
    cs = 256 * 1024  # include/brle/brle.h:8
    return Encoded("brle", cont[hdr + 8:].copy(), total, n_ptr - 1, cs, {"ptr": ptr}, {"container": cont})


# ---------------------------------------------------------------------------
# metadata sidecar (utils.h:46-119)
# ---------------------------------------------------------------------------

def write_meta(path, blobs: list[np.ndarray]) -> None:
    """<path>.meta = [u64 num][u64 lens[num]][blob 0][blob 1]..."""
    raw = [np.ascontiguousarray(b).view(np.uint8).reshape(-1) for b in blobs]
    with open(str(path) + ".meta", "wb") as f:
        f.write(_u64(len(raw)))
        f.write(_u64([r.size for r in raw]))
        for r in raw:
            f.write(r.tobytes())


def read_meta(path) -> list[np.ndarray]:
    m = np.fromfile(str(path) + ".meta", dtype=np.uint8)
    num = int(m[:8].view(np.uint64)[0])
    lens = m[8:8 + 8 * num].view(np.uint64)
    out, off = [], 8 + 8 * num
    for n in lens:
        out.append(m[off:off + int(n)].copy())
        off += int(n)
    return out


def write_lzss(enc: Encoded, path) -> None:
    """lzss::compress_gpu's outputs: the blocks and the .meta sidecar."""
    Path(path).write_bytes(enc.data.tobytes())
    m = enc.meta
    write_meta(path, [np.array([enc.chunk_size], np.uint64), m["blk_off"], m["col_len"], m["col_map"]])


def read_lzss(path) -> Encoded:
    cs, blk, col, cmap = read_meta(path)
    chunk = int(cs.view(np.uint64)[0])
    blk = blk.view(np.uint64)
    n = blk.size - 1
    data = np.fromfile(path, dtype=np.uint8)
    # the reference's containers hold whole chunks (lzss_gpu2.h:1959)
    return Encoded("lzss", data, n * chunk, n, chunk,
                   {"blk_off": blk, "col_len": col.view(np.uint64), "col_map": cmap}, {})


# ---------------------------------------------------------------------------
# RLE v1: data file + side files
# ---------------------------------------------------------------------------

def write_rlev1(enc: Encoded, path, side_dir) -> None:
    side = Path(side_dir)
    side.mkdir(parents=True, exist_ok=True)
    with open(path, "wb") as f:
        f.write(_u64(enc.n_out))
        f.write(enc.data.tobytes())
    enc.meta["col_len"].astype(np.uint64).tofile(side / "rle_v1_col_len.bin")
    enc.meta["blk_off"].astype(np.uint64).tofile(side / "rle_v1_blk_offset.bin")


def read_rlev1(path, side_dir, chunk_size: int = 128 * 1024, comp_col_len: int = 128,
               elem_bytes: int = 4) -> Encoded:
    side = Path(side_dir)
    raw = np.fromfile(path, dtype=np.uint8)
    total = int(raw[:8].view(np.uint64)[0])
    col = _read_u64(side / "rle_v1_col_len.bin")
    blk = _read_u64(side / "rle_v1_blk_offset.bin")
    return Encoded("rlev1", raw[8:].copy(), total, blk.size - 1, chunk_size, {"blk_off": blk, "col_len": col},
                   {"comp_col_len": comp_col_len, "elem_bytes": elem_bytes})


# ---------------------------------------------------------------------------
# flag-byte RLE (1- and 4-byte symbols): blocks + side files
# ---------------------------------------------------------------------------

def write_brle_trans(enc: Encoded, path, side_dir) -> None:
    side = Path(side_dir)
    side.mkdir(parents=True, exist_ok=True)
    Path(path).write_bytes(enc.data.tobytes())
    enc.meta["col_len"].astype(np.uint64).tofile(side / "col_len.bin")
    enc.meta["col_map"].astype(np.uint8).tofile(side / "col_map.bin")
    enc.meta["blk_off"].astype(np.uint64).tofile(side / "blk_offset.bin")


def read_brle_trans(path, side_dir, chunk_size: int = 4096, symbol_bytes: int = 1) -> Encoded:
    """symbol_bytes 1: brle_trans (4 KiB chunks); 4: brle_gpu_4B.h (8 KiB).
    The output is whole chunks, as the reference's decompress_gpu returns."""
    side = Path(side_dir)
    blk = _read_u64(side / "blk_offset.bin")
    n = blk.size - 1
    return Encoded("brle_trans" if symbol_bytes == 1 else "brle_trans4", np.fromfile(path, dtype=np.uint8),
                   n * chunk_size, n, chunk_size,
                   {"blk_off": blk, "col_len": _read_u64(side / "col_len.bin"),
                    "col_map": np.fromfile(side / "col_map.bin", dtype=np.uint8)}, {})


# ---------------------------------------------------------------------------
# Deflate triple and the cuDF single file
# ---------------------------------------------------------------------------

def _uniform_chunk(enc: Encoded) -> int:
    oo = enc.meta["out_off"].astype(np.int64)
    sizes = np.diff(oo)
    cs = int(sizes[0])
    if enc.n_chunks == 0 or not (sizes[:-1] == cs).all() or not 0 < sizes[-1] <= cs:
        raise ValueError("the reference's Deflate layouts hold one uniform chunk size")
    return cs


def write_deflate_triple(enc: Encoded, prefix) -> None:
    """<prefix>_comp.bin, _col_len.bin, _blk_offset.bin (orig_compressor.py:44-126)."""
    _uniform_chunk(enc)
    if enc.params.get("zlib_header", 1) != 1:
        raise ValueError("the triple holds zlib streams")
    p = str(prefix)
    Path(p + "_comp.bin").write_bytes(enc.data.tobytes())
    enc.meta["comp_len"].astype(np.uint64).tofile(p + "_col_len.bin")
    with open(p + "_blk_offset.bin", "wb") as f:
        f.write(_u64(enc.n_out))
        f.write(enc.meta["comp_off"].astype(np.uint64).tobytes())


def read_deflate_triple(prefix, chunk_size: int = 128 * 1024) -> Encoded:
    """num_blk = blk_bytes / 8 - 2 (zlib.h:970); chunk c covers output
    [c * chunk_size, ...), the total truncating the last one."""
    p = str(prefix)
    blk = _read_u64(p + "_blk_offset.bin")
    total, coff = int(blk[0]), blk[1:].copy()
    n = coff.size - 1
    clen = _read_u64(p + "_col_len.bin")[:n]
    oo = np.minimum(np.arange(n + 1, dtype=np.uint64) * np.uint64(chunk_size), np.uint64(total))
    return Encoded("deflate", np.fromfile(p + "_comp.bin", dtype=np.uint8), total, n, 0,
                   {"comp_off": coff, "comp_len": clen, "out_off": oo}, {"zlib_header": 1})


def write_cudf_single(raw, path, chunk_size: int = 64 * 1024, level: int = 9) -> None:
    """rapids_compressor.py:222-280: the column zero-padded to whole chunks,
    each chunk compressed by zlib at `level`, written as
    [u64 chunk_size][u64 n][u64 len[n]][streams] (streams unpadded)."""
    import zlib
    b = np.ascontiguousarray(raw).view(np.uint8).reshape(-1)
    n = (b.size + chunk_size - 1) // chunk_size
    padded = np.zeros(n * chunk_size, np.uint8)
    padded[:b.size] = b
    streams = [zlib.compress(padded[c * chunk_size:(c + 1) * chunk_size].tobytes(), level) for c in range(n)]
    with open(path, "wb") as f:
        f.write(_u64([chunk_size, n]))
        f.write(_u64([len(z) for z in streams]))
        for z in streams:
            f.write(z)


def read_cudf_single(path, total: int) -> Encoded:
    """The file as an Encoded container for the library's decoders.  The
    format does not record the column's length -- the cuDF reader learns it
    from the last stream's bytes_written (base_deflate.h:94-98; see
    decode_cudf_single) -- so it is given here."""
    h = _read_u64(path, count=2)
    cs, n = int(h[0]), int(h[1])
    lens = _read_u64(path, count=n, offset=16)
    data = np.fromfile(path, dtype=np.uint8, offset=16 + 8 * n)
    coff = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    oo = np.minimum(np.arange(n + 1, dtype=np.uint64) * np.uint64(cs), np.uint64(total))
    return Encoded("deflate", data, int(total), n, 0, {"comp_off": coff, "comp_len": lens.copy(), "out_off": oo},
                   {"zlib_header": 1})


def decode_cudf_single(path, device="cuda") -> np.ndarray:
    """base_deflate.h:42-119 over gd_gpuinflate: every stream (its 2-byte zlib
    header skipped) inflated into a chunk_size slot, and the output is
    (n - 1) * chunk_size + the last stream's bytes_written."""
    import ctypes as C
    import torch
    from ._lib import lib
    from .codecs import DecodeError
    h = _read_u64(path, count=2)
    cs, n = int(h[0]), int(h[1])
    lens = _read_u64(path, count=n, offset=16).astype(np.int64)
    data = np.fromfile(path, dtype=np.uint8, offset=16 + 8 * n)
    dev = torch.device(device)
    d_in = torch.from_numpy(np.concatenate([data, np.zeros(16, np.uint8)])).to(dev)
    d_out = torch.empty(max(n * cs, 1), dtype=torch.uint8, device=dev)
    off = np.concatenate([[0], np.cumsum(lens)])
    desc = np.zeros((n, 4), np.uint64)  # gd_inflate_input: src, src_len, dst, dst_len
    desc[:, 0] = d_in.data_ptr() + off[:-1] + 2
    desc[:, 1] = lens - 2
    desc[:, 2] = d_out.data_ptr() + np.arange(n, dtype=np.uint64) * np.uint64(cs)
    desc[:, 3] = cs
    d_desc = torch.from_numpy(desc.view(np.uint8).reshape(-1).copy()).to(dev)
    d_stat = torch.zeros(2 * n, dtype=torch.int64, device=dev)  # gd_inflate_status: bytes_written, status
    s = torch.cuda.current_stream(dev).cuda_stream
    rc = lib().gd_gpuinflate(C.c_void_p(d_desc.data_ptr()), C.c_void_p(d_stat.data_ptr()), n, 0, C.c_void_p(s))
    if rc != 0:
        raise DecodeError(rc, "gd_gpuinflate")
    st = d_stat.cpu().numpy().reshape(n, 2)
    bad = (st[:, 1] & 0xffffffff) != 0
    if bad.any():
        raise DecodeError(int(st[bad][0, 1] & 0xffffffff), "gd_gpuinflate stream")
    total = (n - 1) * cs + int(st[-1, 0])
    return d_out[:total].cpu().numpy()
