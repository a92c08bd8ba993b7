"""GPU tests of the cuDF-shaped Deflate calls and of the bounded hand-off
wait of the decoder/writer pairs:

* gzip members (RFC 1952 headers with and without FEXTRA / FNAME / FCOMMENT /
  FHCRC) through gd_inflate(zlib_header = 2) and through gd_gpuinflate with
  parse_hdr = 1 (cudf::io::gpuinflate, cudf_deflate.cuh:1180-1216,1399-1407),
  against zlib (the oracle) and the input;
* raw deflate through gd_gpuinflate(parse_hdr = 0) at the unaligned source
  pointers a cuDF reader hands it (base_deflate.h:68-72 passes srcDevice + 2);
* gd_copy_uncompressed_blocks (cudf_deflate.cuh:1349-1392,1409-1415) over
  unaligned sources and destinations, copying min(srcSize, dstSize) bytes;
* the decoder/writer hand-off wait running out: with the writer warp told to
  leave early and a short poll limit, every affected stream reports
  GD_ERR_TIMEOUT, the kernel returns, and the next launch on the same
  context decodes bit-exact."""
import ctypes as C
import struct
import zlib

import numpy as np
import pytest

import compression_b200.codecs as cc
import oracle
from compression_b200._lib import lib

pytestmark = pytest.mark.gpu

TIMEOUT = 4  # GD_ERR_TIMEOUT
TUNE_INFLATE_VARIANT, TUNE_PAIR_SPIN, TUNE_WRITER_STOP = 0, 5, 6


def _gzip_member(raw: bytes, flags: int, level: int = 6) -> bytes:
    """One gzip member (RFC 1952) with the optional header fields `flags`
    selects: FHCRC 2, FEXTRA 4, FNAME 8, FCOMMENT 16."""
    hdr = bytearray([0x1F, 0x8B, 8, flags]) + struct.pack("<I", 0x5F5E0F00) + bytes([0, 3])
    if flags & 4:
        extra = b"AB" + struct.pack("<H", 5) + b"xyzzy"
        hdr += struct.pack("<H", len(extra)) + extra
    if flags & 8:
        hdr += b"column_07.bin\x00"
    if flags & 16:
        hdr += b"written by the gzip member builder\x00"
    if flags & 2:
        hdr += struct.pack("<H", zlib.crc32(bytes(hdr)) & 0xFFFF)
    co = zlib.compressobj(level, zlib.DEFLATED, -15)
    body = co.compress(raw) + co.flush()
    return bytes(hdr) + body + struct.pack("<II", zlib.crc32(raw), len(raw) & 0xFFFFFFFF)


def _members(seed: int, n: int):
    rng = np.random.default_rng(seed)
    src = cc.gen_markov_copy(seed, 3 << 20, 32768)
    sizes = rng.integers(1, 400000, n)
    sizes[0] = 700000
    raws, mem, at = [], [], 0
    for i, sz in enumerate(sizes):
        r = src[at % (src.size - int(sz)):][:int(sz)].tobytes()
        at += int(sz)
        raws.append(r)
        mem.append(_gzip_member(r, [0, 8, 4 | 16, 2 | 4 | 8 | 16, 2][i % 5], level=[6, 1, 9, 0][i % 4]))
    return raws, mem


def _container(raws, streams, zlib_header):
    """The Deflate container layout: streams 8-byte padded, back to back."""
    comp_off, data = [0], bytearray()
    for s in streams:
        data += s + bytes((-len(s)) % 8)
        comp_off.append(len(data))
    out_off = np.concatenate([[0], np.cumsum([len(r) for r in raws])]).astype(np.uint64)
    return cc.Encoded("deflate", np.frombuffer(bytes(data), np.uint8).copy(), int(out_off[-1]), len(streams), 0,
                      {"comp_off": np.array(comp_off, np.uint64),
                       "comp_len": np.array([len(s) for s in streams], np.uint64), "out_off": out_off},
                      {"zlib_header": zlib_header})


def test_inflate_gzip_members(cuda):
    import torch
    raws, mem = _members(61, 23)
    enc = _container(raws, mem, 2)
    rc, ref = oracle.decode(enc)
    assert rc == 0 and ref.tobytes() == b"".join(raws)
    job = cc.DeviceJob(enc, cuda)
    job.launch()
    torch.cuda.synchronize()
    assert (job.status() == 0).all(), job.status()
    assert np.array_equal(job.output(), ref)
    # a member whose magic is wrong is reported, the others still decode
    bad = bytearray(mem[3])
    bad[1] = 0x8C
    enc2 = _container(raws, mem[:3] + [bytes(bad)] + mem[4:], 2)
    job = cc.DeviceJob(enc2, cuda)
    job.launch()
    torch.cuda.synchronize()
    st = job.status()
    assert st[3] == 2 and (np.delete(st, 3) == 0).all(), st


def _descs(torch, dev, srcs, dsts_cap, src_shift=0, dst_shift=0):
    """cuDF input descriptors over one device source arena and one output
    arena; every source starts src_shift bytes past an 8-byte boundary."""
    so, sbuf = [], bytearray()
    for s in srcs:
        sbuf += bytes((-len(sbuf)) % 8) + bytes(src_shift)
        so.append(len(sbuf))
        sbuf += s
    sbuf += bytes(64)
    d_src = torch.from_numpy(np.frombuffer(bytes(sbuf), np.uint8).copy()).to(dev)
    do = np.concatenate([[0], np.cumsum([c + 16 for c in dsts_cap])]).astype(np.int64)
    d_dst = torch.full((int(do[-1]) + 64,), 0xEE, dtype=torch.uint8, device=dev)
    desc = np.zeros((len(srcs), 4), np.uint64)
    for i, s in enumerate(srcs):
        desc[i] = [d_src.data_ptr() + so[i], len(s), d_dst.data_ptr() + int(do[i]) + dst_shift, dsts_cap[i]]
    d_desc = torch.from_numpy(desc.view(np.int64).reshape(-1)).to(dev)
    return d_src, d_dst, d_desc, do


def _stream_ptr(torch):
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


@pytest.mark.parametrize("shift", [0, 3])
def test_gpuinflate_parse_hdr_gzip(cuda, shift):
    import torch
    raws, mem = _members(62 + shift, 17)
    cap = [len(r) + 1000 for r in raws]  # dstSize is a capacity
    d_src, d_dst, d_desc, do = _descs(torch, cuda, mem, cap, src_shift=shift)
    d_stat = torch.full((len(mem) * 2,), -1, dtype=torch.int64, device=cuda)
    rc = lib().gd_gpuinflate(C.c_void_p(d_desc.data_ptr()), C.c_void_p(d_stat.data_ptr()), len(mem), 1,
                             _stream_ptr(torch))
    assert rc == 0
    torch.cuda.synchronize()
    st = d_stat.cpu().numpy().reshape(-1, 2)
    out = d_dst.cpu().numpy()
    for i, r in enumerate(raws):
        assert int(st[i, 0]) == len(r), i                      # bytes_written
        assert int(st[i, 1]) & 0xFFFFFFFF == 0, i               # status
        assert out[int(do[i]):int(do[i]) + len(r)].tobytes() == r, i


def test_gpuinflate_raw_deflate_unaligned(cuda):
    """The cuDF reader's flow: zlib streams handed over past their 2-byte
    header (srcDevice + 2), i.e. raw deflate at unaligned addresses."""
    import torch
    raws, _ = _members(63, 11)
    zs = [zlib.compress(r, 6)[2:] for r in raws]
    d_src, d_dst, d_desc, do = _descs(torch, cuda, zs, [len(r) for r in raws], src_shift=2)
    d_stat = torch.full((len(zs) * 2,), -1, dtype=torch.int64, device=cuda)
    assert lib().gd_gpuinflate(C.c_void_p(d_desc.data_ptr()), C.c_void_p(d_stat.data_ptr()), len(zs), 0,
                               _stream_ptr(torch)) == 0
    torch.cuda.synchronize()
    st = d_stat.cpu().numpy().reshape(-1, 2)
    out = d_dst.cpu().numpy()
    for i, r in enumerate(raws):
        assert int(st[i, 0]) == len(r) and int(st[i, 1]) & 0xFFFFFFFF == 0, i
        assert out[int(do[i]):int(do[i]) + len(r)].tobytes() == r, i


def test_copy_uncompressed_blocks(cuda):
    import torch
    rng = np.random.default_rng(64)
    sizes = [0, 1, 3, 31, 32, 33, 4097, (1 << 20) + 3, 100000]
    srcs = [rng.integers(0, 256, n).astype(np.uint8).tobytes() for n in sizes]
    caps = list(sizes)
    caps[-1] = 77777  # dstSize below srcSize: min(srcSize, dstSize) bytes are copied
    for sshift, dshift in [(0, 0), (1, 3), (5, 2)]:
        d_src, d_dst, d_desc, do = _descs(torch, cuda, srcs, caps, src_shift=sshift, dst_shift=dshift)
        assert lib().gd_copy_uncompressed_blocks(C.c_void_p(d_desc.data_ptr()), len(srcs), _stream_ptr(torch)) == 0
        torch.cuda.synchronize()
        out = d_dst.cpu().numpy()
        for i, s in enumerate(srcs):
            n = min(len(s), caps[i])
            o = int(do[i]) + dshift
            assert out[o:o + n].tobytes() == s[:n], (i, sshift, dshift)
            assert (out[int(do[i]):o] == 0xEE).all() and out[o + n] == 0xEE, (i, sshift, dshift)


@pytest.mark.parametrize("variant", [6, 12])
def test_pair_wait_runs_out(cuda, variant):
    import torch
    raw = cc.gen_markov_copy(65, 3 << 20, 32768)
    oo = np.array([0, 1 << 20, (1 << 20) + 300000, 2 << 20, 3 << 20], np.uint64)
    enc = cc.deflate_encode(raw, oo, 6)
    L = lib()
    prev = [L.gd_tune_set(k, v) for k, v in
            ((TUNE_INFLATE_VARIANT, variant), (TUNE_PAIR_SPIN, 2048), (TUNE_WRITER_STOP, 1))]
    try:
        job = cc.DeviceJob(enc, cuda)
        job.launch()
        torch.cuda.synchronize()  # the kernel returned: every wait was bounded
        st = job.status()
    finally:
        for k, v in zip((TUNE_INFLATE_VARIANT, TUNE_PAIR_SPIN, TUNE_WRITER_STOP), prev):
            L.gd_tune_set(k, v)
    assert (st == TIMEOUT).all(), st
    # the context is still usable: the same streams decode bit-exact
    L.gd_tune_set(TUNE_INFLATE_VARIANT, variant)
    try:
        job = cc.DeviceJob(enc, cuda)
        job.launch()
        torch.cuda.synchronize()
        assert (job.status() == 0).all()
        assert np.array_equal(job.output(), raw)
    finally:
        L.gd_tune_set(TUNE_INFLATE_VARIANT, prev[0])
