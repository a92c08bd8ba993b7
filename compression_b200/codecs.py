"""Host-side mirror of the reference's codec interface over the C ABI.

Each codec has an encoder (host, produces the reference container) and a
device job that owns the device copies of the container and launches the
sm_100a decoder through the C ABI.  torch provides device memory and streams
only; all decoding happens in libgd.so.

Reference interfaces mirrored (ZaidQureshi/compression):
  brle::compress_gpu / decompress_gpu          include/brle/brle.h:251-342
  rle_v1::compress_gpu / decompress_gpu        include/rle_v1/rlev1.h:25-199
  rlev2::compress_gpu_transpose / decompress_gpu
                                               include/rlev2/encoder_trans.h:428-537,
                                               include/rlev2/decoder_trans.h:615-681
  lzss::compress_gpu / decompress_gpu          include/lzss/lzss_gpu2.h:1915-2314
  deflate::decompress_gpu (+ Python producer)  include/zlib/zlib.h:966-1082,
                                               orig_compressor.py:44-126
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from ._lib import lib

BRLE_CHUNK = 256 * 1024  # include/brle/brle.h:8


class DecodeError(RuntimeError):
    def __init__(self, status: int, where: str = ""):
        s = lib().gd_status_string(int(status)).decode()
        super().__init__(f"{where}: {s} ({status})")
        self.status = int(status)


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def check(rc: int, where: str) -> None:
    if rc != 0:
        raise DecodeError(rc, where)


# --------------------------------------------------------------------------
# generators
# --------------------------------------------------------------------------

def gen_rlev1_ints(seed: int, n: int) -> np.ndarray:
    a = np.empty(n, dtype=np.int32)
    lib().gd_gen_rlev1_ints(seed, n, _p(a))
    return a


def gen_brle_bytes(seed: int, n: int) -> np.ndarray:
    a = np.empty(n, dtype=np.uint8)
    lib().gd_gen_brle_bytes(seed, n, _p(a))
    return a


def gen_rlev2_ints(seed: int, n: int) -> np.ndarray:
    a = np.empty(n, dtype=np.int64)
    lib().gd_gen_rlev2_ints(seed, n, _p(a))
    return a


def gen_markov_copy(seed: int, n: int, max_dist: int) -> np.ndarray:
    a = np.empty(n, dtype=np.uint8)
    lib().gd_gen_markov_copy(seed, n, max_dist, _p(a))
    return a


def loguniform_sizes(seed: int, n: int, lo: int, hi: int, total: int, granule: int = 1) -> np.ndarray:
    a = np.empty(n, dtype=np.uint64)
    check(lib().gd_gen_loguniform_sizes(seed, n, lo, hi, total, granule, _p(a)), "loguniform_sizes")
    return a


# --------------------------------------------------------------------------
# encoded containers
# --------------------------------------------------------------------------

@dataclass
class Encoded:
    """One compressed column: payload bytes plus its metadata arrays."""
    codec: str
    data: np.ndarray                  # uint8 payload (blocks / chunk streams)
    n_out: int                        # decompressed bytes
    n_chunks: int
    chunk_size: int = 0
    meta: dict = field(default_factory=dict)   # named uint64/uint8 arrays
    params: dict = field(default_factory=dict)

    @property
    def comp_bytes(self) -> int:
        return int(self.data.nbytes)

    @property
    def meta_bytes(self) -> int:
        return int(sum(v.nbytes for v in self.meta.values()))


def _as_u8(raw) -> np.ndarray:
    a = np.ascontiguousarray(raw)
    return a.view(np.uint8).reshape(-1)


def brle_encode(raw, chunk_size: int = BRLE_CHUNK) -> Encoded:
    """brle::compress_gpu: container [u32 n_ptr][u64 ptr[n_ptr]][u64 total][data]."""
    b = _as_u8(raw)
    L = lib()
    cap = L.gd_brle_max_encoded_bytes(b.size, chunk_size)
    out = np.empty(cap, dtype=np.uint8)
    n = L.gd_brle_encode(_p(b), b.size, chunk_size, _p(out))
    if n == 0:
        raise ValueError("brle encode failed")
    cont = out[:n].copy()
    n_ptr = int(cont[:4].view(np.uint32)[0])
    ptr = cont[4:4 + 8 * n_ptr].copy().view(np.uint64)
    hdr = 4 + 8 * n_ptr + 8
    return Encoded("brle", cont[hdr:].copy(), b.size, n_ptr - 1, chunk_size, {"ptr": ptr}, {"container": cont})


def brle_container(enc: Encoded) -> np.ndarray:
    return enc.params["container"]


def rlev1_encode(raw, chunk_size: int = 128 * 1024, comp_col_len: int = 128, elem_bytes: int = 4) -> Encoded:
    """rle_v1::compress_gpu (32-lane interleaved blocks + col_len + blk_offset)."""
    b = _as_u8(raw)
    L = lib()
    nc = (b.size + chunk_size - 1) // chunk_size
    cap = L.gd_rlev1_max_encoded_bytes(b.size, chunk_size)
    data = np.empty(cap, dtype=np.uint8)
    blk = np.empty(nc + 1, dtype=np.uint64)
    col = np.empty(32 * nc, dtype=np.uint64)
    n = L.gd_rlev1_encode(_p(b), b.size, chunk_size, comp_col_len, elem_bytes, _p(data), _p(blk), _p(col))
    if n == 0:
        raise ValueError("rlev1 encode failed")
    return Encoded("rlev1", data[:n].copy(), b.size, nc, chunk_size, {"blk_off": blk, "col_len": col},
                   {"comp_col_len": comp_col_len, "elem_bytes": elem_bytes})


def rlev2_encode(raw, chunk_size: int = 256 * 1024, read_unit: int = 32) -> Encoded:
    """rlev2::compress_gpu_transpose (8-byte values)."""
    b = _as_u8(raw)
    L = lib()
    nc = (b.size + chunk_size - 1) // chunk_size
    cap = L.gd_rlev2_max_encoded_bytes(b.size, chunk_size)
    data = np.empty(cap, dtype=np.uint8)
    blk = np.empty(nc + 1, dtype=np.uint64)
    col = np.empty(32 * nc, dtype=np.uint64)
    n = L.gd_rlev2_encode(_p(b), b.size, chunk_size, read_unit, _p(data), _p(blk), _p(col))
    if n == 0:
        raise ValueError("rlev2 encode failed")
    return Encoded("rlev2", data[:n].copy(), b.size, nc, chunk_size, {"blk_off": blk, "col_len": col},
                   {"read_unit": read_unit})


def lzss_encode(raw, chunk_size: int = 64 * 1024) -> Encoded:
    """lzss::compress_gpu (32-column interleaved blocks + .meta arrays)."""
    b = _as_u8(raw)
    L = lib()
    nc = (b.size + chunk_size - 1) // chunk_size
    cap = L.gd_lzss_max_encoded_bytes(b.size, chunk_size)
    data = np.empty(cap, dtype=np.uint8)
    blk = np.empty(nc + 1, dtype=np.uint64)
    col = np.empty(32 * nc, dtype=np.uint64)
    cmap = np.empty(32 * nc, dtype=np.uint8)
    n = L.gd_lzss_encode(_p(b), b.size, chunk_size, _p(data), _p(blk), _p(col), _p(cmap))
    if n == 0:
        raise ValueError("lzss encode failed")
    return Encoded("lzss", data[:n].copy(), b.size, nc, chunk_size,
                   {"blk_off": blk, "col_len": col, "col_map": cmap}, {})


def lzss_contig_encode(raw, chunk_size: int = 128 * 1024) -> Encoded:
    """lzss::compress_gpu, contiguous container (include/lzss/lzss.h:1060-1124):
    one token stream per chunk.  params["container"] is the whole file."""
    b = _as_u8(raw)
    L = lib()
    cap = L.gd_lzss_contig_max_encoded_bytes(b.size, chunk_size)
    cont = np.empty(cap, dtype=np.uint8)
    n = L.gd_lzss_contig_encode(_p(b), b.size, chunk_size, _p(cont))
    if n == 0:
        raise ValueError("lzss contiguous encode failed")
    cont = cont[:n].copy()
    nc = (b.size + chunk_size - 1) // chunk_size
    ends = cont[28:28 + 8 * nc].copy().view(np.uint64)
    return Encoded("lzss_contig", cont[28 + 8 * nc:].copy(), b.size, nc, chunk_size, {"ends": ends},
                   {"container": cont})


def brle_trans_encode(raw, chunk_size: int = 4096) -> Encoded:
    """brle_trans::compress_gpu (include/brle/brle_trans.h:563-660): flag-byte
    byte-RLE columns in the ranked 32-column layout + side-file arrays."""
    b = _as_u8(raw)
    L = lib()
    nc = (b.size + chunk_size - 1) // chunk_size
    cap = L.gd_brle_trans_max_encoded_bytes(b.size, chunk_size)
    data = np.empty(cap, dtype=np.uint8)
    blk = np.empty(nc + 1, dtype=np.uint64)
    col = np.empty(32 * nc, dtype=np.uint64)
    cmap = np.empty(32 * nc, dtype=np.uint8)
    n = L.gd_brle_trans_encode(_p(b), b.size, chunk_size, _p(data), _p(blk), _p(col), _p(cmap))
    if n == 0:
        raise ValueError("brle_trans encode failed")
    return Encoded("brle_trans", data[:n].copy(), b.size, nc, chunk_size,
                   {"blk_off": blk, "col_len": col, "col_map": cmap}, {})


def brle_trans4_encode(raw, chunk_size: int = 8192) -> Encoded:
    """brle::compress_gpu of include/brle/brle_gpu_4B.h:640-715: the flag-byte
    columns over 4-byte symbols, same ranked 32-column layout (8 KiB chunks
    in the reference)."""
    b = _as_u8(raw)
    L = lib()
    nc = (b.size + chunk_size - 1) // chunk_size
    cap = L.gd_brle_trans4_max_encoded_bytes(b.size, chunk_size)
    data = np.empty(cap, dtype=np.uint8)
    blk = np.empty(nc + 1, dtype=np.uint64)
    col = np.empty(32 * nc, dtype=np.uint64)
    cmap = np.empty(32 * nc, dtype=np.uint8)
    n = L.gd_brle_trans4_encode(_p(b), b.size, chunk_size, _p(data), _p(blk), _p(col), _p(cmap))
    if n == 0:
        raise ValueError("brle_trans4 encode failed")
    return Encoded("brle_trans4", data[:n].copy(), b.size, nc, chunk_size,
                   {"blk_off": blk, "col_len": col, "col_map": cmap}, {})


def deflate_encode(raw, out_off: np.ndarray, level: int = 6, mode: np.ndarray | None = None,
                   zlib_header: int = 1) -> Encoded:
    """Per-chunk zlib streams padded to 8 bytes (orig_compressor.py:44-126).

    out_off[n+1]: chunk c covers raw[out_off[c]:out_off[c+1]].  mode[c]:
    0 default strategy, 1 fixed Huffman (Z_FIXED), 2 stored (level 0)."""
    b = _as_u8(raw)
    L = lib()
    oo = np.ascontiguousarray(out_off, dtype=np.uint64)
    n = oo.size - 1
    cap = L.gd_deflate_max_encoded_bytes(_p(oo), n)
    data = np.empty(cap, dtype=np.uint8)
    coff = np.empty(n + 1, dtype=np.uint64)
    clen = np.empty(n, dtype=np.uint64)
    m = None if mode is None else np.ascontiguousarray(mode, dtype=np.uint8)
    got = L.gd_deflate_encode(_p(b), _p(oo), n, level, None if m is None else _p(m), zlib_header, _p(data),
                              _p(coff), _p(clen))
    if got == 0:
        raise ValueError("deflate encode failed")
    return Encoded("deflate", data[:got].copy(), int(oo[-1]), n, 0,
                   {"comp_off": coff, "comp_len": clen, "out_off": oo}, {"zlib_header": zlib_header})


# --------------------------------------------------------------------------
# device encoders (byte-RLE / LZSS / RLE v1 / RLE v2 containers written on the GPU)
# --------------------------------------------------------------------------

def encode_device(codec: str, d_col, chunk_size: int, *, comp_col_len: int = 128, elem_bytes: int = 4,
                  read_unit: int = 32, stream=None, bufs: dict | None = None) -> dict:
    """Enqueue gd_rlev1_encode_device / gd_rlev2_encode_device /
    gd_lzss_encode_device on `d_col`, a CUDA uint8 tensor holding the column.
    Returns the device tensors {"data", "blk_off", "col_len", "col_map"
    (LZSS), "status", "scratch"}; "data" is sized to
    the bound and the container's length is blk_off[-1].  `bufs` (a previous
    return value) reuses its buffers.  For "brle" (gd_brle_encode_device) the
    tensors are {"container", "size", "scratch"}: the whole container and its
    length."""
    import torch
    n = int(d_col.numel())
    L = lib()
    if codec == "brle":
        return _brle_encode_device(d_col, chunk_size, stream, bufs)
    if codec == "rlev1":
        bound = L.gd_rlev1_encode_bound(n, chunk_size, elem_bytes)
    elif codec == "lzss":
        bound = L.gd_lzss_encode_bound(n, chunk_size)
    elif codec == "brle_trans":
        bound = L.gd_brle_trans_encode_bound(n, chunk_size)
    elif codec == "rlev2":
        bound = L.gd_rlev2_encode_bound(n, chunk_size)
    else:
        raise ValueError(f"no device encoder for {codec}")
    if bound == 0:
        raise ValueError("bad encoder arguments")
    nc = (n + chunk_size - 1) // chunk_size
    dev = d_col.device
    if bufs is None or bufs["data"].numel() < bound or bufs["blk_off"].numel() != nc + 1:
        bufs = {"scratch": torch.empty(bound, dtype=torch.uint8, device=dev),
                "data": torch.empty(bound, dtype=torch.uint8, device=dev),
                "blk_off": torch.empty(nc + 1, dtype=torch.int64, device=dev),
                "col_len": torch.empty(32 * nc, dtype=torch.int64, device=dev),
                "status": torch.empty(nc, dtype=torch.int32, device=dev),
                "col_map": torch.empty(32 * nc, dtype=torch.uint8, device=dev)}
    s = (stream or torch.cuda.current_stream()).cuda_stream
    p = lambda t: C.c_void_p(t.data_ptr())
    if codec == "rlev1":
        rc = L.gd_rlev1_encode_device(p(d_col), n, chunk_size, comp_col_len, elem_bytes, p(bufs["scratch"]),
                                      p(bufs["data"]), p(bufs["blk_off"]), p(bufs["col_len"]), p(bufs["status"]),
                                      C.c_void_p(s))
    elif codec in ("lzss", "brle_trans"):
        fn = L.gd_lzss_encode_device if codec == "lzss" else L.gd_brle_trans_encode_device
        rc = fn(p(d_col), n, chunk_size, p(bufs["scratch"]), p(bufs["data"]), p(bufs["blk_off"]),
                p(bufs["col_len"]), p(bufs["col_map"]), p(bufs["status"]), C.c_void_p(s))
    else:
        rc = L.gd_rlev2_encode_device(p(d_col), n, chunk_size, read_unit, p(bufs["scratch"]), p(bufs["data"]),
                                      p(bufs["blk_off"]), p(bufs["col_len"]), p(bufs["status"]), C.c_void_p(s))
    check(rc, f"gd_{codec}_encode_device")
    return bufs


def _brle_encode_device(d_col, chunk_size: int, stream=None, bufs: dict | None = None) -> dict:
    """gd_brle_encode_device: {"container", "size" (device int64[1]), "scratch"}."""
    import torch
    n = int(d_col.numel())
    L = lib()
    cap = L.gd_brle_max_encoded_bytes(n, chunk_size)
    sb = L.gd_brle_encode_scratch_bytes(n, chunk_size)
    if sb == 0:
        raise ValueError("bad encoder arguments")
    dev = d_col.device
    if bufs is None or bufs["container"].numel() < cap or bufs["scratch"].numel() < sb:
        bufs = {"scratch": torch.empty(sb, dtype=torch.uint8, device=dev),
                "container": torch.empty(cap, dtype=torch.uint8, device=dev),
                "size": torch.zeros(1, dtype=torch.int64, device=dev)}
    s = (stream or torch.cuda.current_stream()).cuda_stream
    p = lambda t: C.c_void_p(t.data_ptr())
    check(L.gd_brle_encode_device(p(d_col), n, chunk_size, p(bufs["scratch"]), p(bufs["container"]),
                                  p(bufs["size"]), C.c_void_p(s)), "gd_brle_encode_device")
    return bufs


def encode_gpu(codec: str, raw, chunk_size: int, *, comp_col_len: int = 128, elem_bytes: int = 4,
               read_unit: int = 32) -> Encoded:
    """The device encoder from host memory: the same Encoded as brle_encode /
    lzss_encode / rlev1_encode / rlev2_encode (brle::compress_gpu,
    include/brle/brle.h:242-303; lzss::compress_gpu, include/lzss/lzss_gpu2.h:1915-2127;
    rle_v1::compress_gpu, include/rle_v1/rlev1.h:25-97;
    rlev2::compress_gpu_transpose, include/rlev2/encoder_trans.h:428-537)."""
    import torch
    b = _as_u8(raw)
    d = torch.from_numpy(b.copy()).cuda()
    r = encode_device(codec, d, chunk_size, comp_col_len=comp_col_len, elem_bytes=elem_bytes, read_unit=read_unit)
    torch.cuda.synchronize()
    if codec == "brle":
        cont = r["container"][:int(r["size"].item())].cpu().numpy()
        n_ptr = int(cont[:4].view(np.uint32)[0])
        ptr = cont[4:4 + 8 * n_ptr].copy().view(np.uint64)
        hdr = 4 + 8 * n_ptr + 8
        return Encoded("brle", cont[hdr:].copy(), b.size, n_ptr - 1, chunk_size, {"ptr": ptr}, {"container": cont})
    st = r["status"].cpu().numpy()
    if (st != 0).any():
        raise DecodeError(int(st[st != 0][0]), f"gd_{codec}_encode_device")
    blk = r["blk_off"].cpu().numpy().view(np.uint64)
    col = r["col_len"].cpu().numpy().view(np.uint64)
    data = r["data"][:int(blk[-1])].cpu().numpy()
    nc = blk.size - 1
    meta = {"blk_off": blk, "col_len": col}
    if codec in ("lzss", "brle_trans"):
        meta["col_map"] = r["col_map"].cpu().numpy()
    params = ({"comp_col_len": comp_col_len, "elem_bytes": elem_bytes} if codec == "rlev1"
              else {"read_unit": read_unit} if codec == "rlev2" else {})
    return Encoded(codec, data, b.size, nc, chunk_size, meta, params)


def _take(ptr: C.c_void_p, n: int, dtype=np.uint8) -> np.ndarray:
    """Copy a library-owned host buffer into numpy and release it (gd_free)."""
    a = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_uint8)), shape=(n,)).copy() if n else np.empty(0, np.uint8)
    lib().gd_free(ptr)
    return a.view(dtype)


def compress_host(codec: str, raw, chunk_size: int = 0, *, comp_col_len: int = 128, elem_bytes: int = 4,
                  read_unit: int = 32) -> Encoded:
    """The reference-shaped synchronous compress call (H2D, device encoder,
    D2H) via the C ABI: gd_brle_compress (256 KiB chunks, brle::compress_gpu),
    gd_rlev1_compress (rle_v1::compress_gpu), gd_rlev2_compress
    (rlev2::compress_gpu_transpose; the Encoded keeps the encoded size in
    blk_off[-1], as the host encoder's does) or gd_lzss_compress (128 KiB
    chunks, lzss::compress_gpu).  chunk_size applies to RLE v1 / v2."""
    b = _as_u8(raw)
    L = lib()
    out, n = C.c_void_p(), C.c_uint64()
    if codec == "brle":
        check(L.gd_brle_compress(_p(b), b.size, C.byref(out), C.byref(n)), "gd_brle_compress")
        cont = _take(out, n.value)
        n_ptr = int(cont[:4].view(np.uint32)[0])
        ptr = cont[4:4 + 8 * n_ptr].copy().view(np.uint64)
        hdr = 4 + 8 * n_ptr + 8
        return Encoded("brle", cont[hdr:].copy(), b.size, n_ptr - 1, BRLE_CHUNK, {"ptr": ptr}, {"container": cont})
    if codec == "lzss":
        meta, lens, num = C.c_void_p(), C.c_void_p(), C.c_uint64()
        check(L.gd_lzss_compress(_p(b), b.size, C.byref(out), C.byref(n), C.byref(meta), C.byref(lens),
                                 C.byref(num)), "gd_lzss_compress")
        data = _take(out, n.value)
        ptrs = C.cast(meta, C.POINTER(C.c_void_p))
        ln = np.ctypeslib.as_array(C.cast(lens, C.POINTER(C.c_uint64)), shape=(num.value,)).copy()
        blobs = [_take(C.c_void_p(ptrs[i]), int(ln[i])) for i in range(num.value)]
        L.gd_free(meta)
        L.gd_free(lens)
        cs = int(blobs[0].view(np.uint64)[0])
        m = {"blk_off": blobs[1].view(np.uint64), "col_len": blobs[2].view(np.uint64), "col_map": blobs[3]}
        return Encoded("lzss", data, b.size, m["blk_off"].size - 1, cs, m, {})
    col, blk, nc = C.c_void_p(), C.c_void_p(), C.c_uint64()
    if codec == "rlev1":
        check(L.gd_rlev1_compress(_p(b), b.size, comp_col_len, elem_bytes, chunk_size, C.byref(out), C.byref(n),
                                  C.byref(col), C.byref(blk), C.byref(nc)), "gd_rlev1_compress")
        cont = _take(out, n.value)
        params = {"comp_col_len": comp_col_len, "elem_bytes": elem_bytes, "container": cont}
        data = cont[8:].copy()
    elif codec == "rlev2":
        check(L.gd_rlev2_compress(_p(b), b.size, read_unit, chunk_size, C.byref(out), C.byref(n), C.byref(blk),
                                  C.byref(col), C.byref(nc)), "gd_rlev2_compress")
        data = _take(out, n.value)
        params = {"read_unit": read_unit}
    else:
        raise ValueError(f"no compress call for {codec}")
    k = nc.value
    bo = _take(blk, 8 * (k + 1), np.uint64)
    if codec == "rlev2":
        assert int(bo[-1]) == b.size  # the reference keeps the column's size there
        bo = bo.copy()
        bo[-1] = data.size
    return Encoded(codec, data, b.size, k, chunk_size, {"blk_off": bo, "col_len": _take(col, 8 * 32 * k, np.uint64)},
                   params)


# --------------------------------------------------------------------------
# device jobs
# --------------------------------------------------------------------------

class DeviceJob:
    """Device-resident copy of an Encoded container plus its output buffer.

    ``launch(stream)`` enqueues the decoder; ``status()`` returns the per-chunk
    status array.  torch is used for allocation and streams only.
    """

    def __init__(self, enc: Encoded, device="cuda", out=None):
        import torch
        self.torch = torch
        self.enc = enc
        self.dev = torch.device(device)
        # payload padded to 16 bytes (the inflate reader fetches aligned words)
        pad = (-enc.data.size) % 16 + 16
        d = np.concatenate([enc.data, np.zeros(pad, dtype=np.uint8)])
        self.d_data = torch.from_numpy(d).to(self.dev)
        self.d_meta = {k: torch.from_numpy(np.ascontiguousarray(v)).to(self.dev) for k, v in enc.meta.items()}
        # bound on the longest lane stream (sizes the decoders' shared memory)
        self.max_lane = int(enc.meta["col_len"].max()) if "col_len" in enc.meta and enc.n_chunks else 0
        out_n = enc.n_out
        if enc.codec == "lzss":
            out_n = enc.n_chunks * enc.chunk_size
        self.out_n = out_n
        self.d_out = out if out is not None else torch.empty(max(out_n, 16), dtype=torch.uint8, device=self.dev)
        self.d_status = torch.zeros(max(enc.n_chunks, 1), dtype=torch.int32, device=self.dev)
        self.d_order = None
        if enc.codec == "deflate" and enc.n_chunks > 1:
            # streams start longest first (the kernel hands them out in this order)
            sizes = np.diff(enc.meta["out_off"].astype(np.int64))
            order = np.argsort(-sizes, kind="stable").astype(np.uint32)
            self.d_order = torch.from_numpy(order).to(self.dev)

    def launch(self, stream=None) -> None:
        L = lib()
        e = self.enc
        s = C.c_void_p(stream.cuda_stream if stream is not None else
                       self.torch.cuda.current_stream(self.dev).cuda_stream)
        m = self.d_meta
        ptr = lambda t: C.c_void_p(t.data_ptr())
        if e.codec == "brle":
            rc = L.gd_brle_decode(ptr(self.d_data), ptr(m["ptr"]), e.n_chunks, e.chunk_size, ptr(self.d_out),
                                  e.n_out, ptr(self.d_status), s)
        elif e.codec == "rlev1":
            rc = L.gd_rlev1_decode(ptr(self.d_data), ptr(m["col_len"]), ptr(m["blk_off"]), e.n_chunks,
                                   e.chunk_size, e.params["comp_col_len"], e.params["elem_bytes"],
                                   ptr(self.d_out), e.n_out, self.max_lane, ptr(self.d_status), s)
        elif e.codec == "rlev2":
            rc = L.gd_rlev2_decode(ptr(self.d_data), ptr(m["col_len"]), ptr(m["blk_off"]), e.n_chunks,
                                   e.chunk_size, e.params["read_unit"], ptr(self.d_out), e.n_out,
                                   self.max_lane, ptr(self.d_status), s)
        elif e.codec == "lzss":
            rc = L.gd_lzss_decode(ptr(self.d_data), ptr(m["blk_off"]), ptr(m["col_len"]), ptr(m["col_map"]),
                                  e.n_chunks, e.chunk_size, ptr(self.d_out), self.out_n, ptr(self.d_status), s)
        elif e.codec == "lzss_contig":
            rc = L.gd_lzss_contig_decode(ptr(self.d_data), ptr(m["ends"]), e.n_chunks, e.chunk_size, ptr(self.d_out),
                                         e.n_out, ptr(self.d_status), s)
        elif e.codec in ("brle_trans", "brle_trans4"):
            fn = L.gd_brle_trans_decode if e.codec == "brle_trans" else L.gd_brle_trans4_decode
            rc = fn(ptr(self.d_data), ptr(m["blk_off"]), ptr(m["col_len"]), ptr(m["col_map"]),
                    e.n_chunks, e.chunk_size, ptr(self.d_out), e.n_out, ptr(self.d_status), s)
        elif e.codec == "deflate" and self.d_order is not None:
            rc = L.gd_inflate_ordered(ptr(self.d_data), ptr(m["comp_off"]), ptr(m["comp_len"]), ptr(m["out_off"]),
                                      e.n_chunks, e.params["zlib_header"], ptr(self.d_out), ptr(self.d_status),
                                      ptr(self.d_order), s)
        elif e.codec == "deflate":
            rc = L.gd_inflate(ptr(self.d_data), ptr(m["comp_off"]), ptr(m["comp_len"]), ptr(m["out_off"]),
                              e.n_chunks, e.params["zlib_header"], ptr(self.d_out), ptr(self.d_status), s)
        else:
            raise ValueError(e.codec)
        check(rc, f"{e.codec} launch")

    def status(self) -> np.ndarray:
        return self.d_status.cpu().numpy().astype(np.uint32)

    def output(self) -> np.ndarray:
        return self.d_out[: self.enc.n_out].cpu().numpy()


_PINNED_KEEP: list = []  # pinned tensors backing the numpy views below


def _pinned_copy(a: np.ndarray) -> np.ndarray:
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    _PINNED_KEEP.append(t)
    return t.numpy()


def decode_host_pinned(enc: Encoded) -> np.ndarray:
    """decode_host with the container held in page-locked host memory (the
    pinned copies are made once and cached on `enc`)."""
    if "_pinned" not in enc.params:
        pm = {k: _pinned_copy(v) for k, v in enc.meta.items()}
        pd = _pinned_copy(enc.data)
        cont = enc.params.get("container")
        if cont is None and enc.codec == "rlev1":
            cont = np.concatenate([np.array([enc.n_out], dtype=np.uint64).view(np.uint8), enc.data])
        pc = _pinned_copy(cont) if cont is not None else None
        enc.params["_pinned"] = (pd, pm, pc)
    pd, pm, pc = enc.params["_pinned"]
    view = Encoded(enc.codec, pd, enc.n_out, enc.n_chunks, enc.chunk_size, pm,
                   {k: v for k, v in enc.params.items() if k not in ("_pinned", "container")})
    if pc is not None:
        view.params["container"] = pc
    return decode_host(view, keep=False)


def decode_host(enc: Encoded, keep: bool = True) -> np.ndarray:
    """Reference-shaped synchronous host call (H2D, decode, D2H) via the C ABI.

    keep=False returns None after releasing the library's output buffer (used
    for timing the call itself)."""
    L = lib()
    out = C.c_void_p()
    n = C.c_uint64()
    m = enc.meta
    if enc.codec == "brle":
        cont = enc.params["container"]
        rc = L.gd_brle_decompress(_p(cont), cont.size, C.byref(out), C.byref(n))
    elif enc.codec == "rlev1":
        buf = enc.params.get("container")  # [u64 decompressed size][blocks], as the reference reads it
        if buf is None:
            buf = np.concatenate([np.array([enc.n_out], dtype=np.uint64).view(np.uint8), enc.data])
        rc = L.gd_rlev1_decompress(_p(buf), buf.size, _p(m["col_len"]), m["col_len"].nbytes, _p(m["blk_off"]),
                                   m["blk_off"].nbytes, enc.params["comp_col_len"], enc.params["elem_bytes"],
                                   enc.chunk_size, C.byref(out), C.byref(n))
    elif enc.codec == "rlev2":
        blk = m["blk_off"].copy()
        blk[-1] = enc.n_out  # the reference stores the decompressed size there
        rc = L.gd_rlev2_decompress(_p(enc.data), enc.data.size, enc.n_chunks, _p(blk), _p(m["col_len"]),
                                   enc.params["read_unit"], enc.chunk_size, C.byref(out), C.byref(n))
    elif enc.codec == "lzss":
        cs = np.array([enc.chunk_size], dtype=np.uint64)
        arrs = [cs, m["blk_off"], m["col_len"], m["col_map"]]
        ptrs = (C.c_void_p * 4)(*[_p(a) for a in arrs])
        lens = np.array([a.nbytes for a in arrs], dtype=np.uint64)
        rc = L.gd_lzss_decompress(_p(enc.data), enc.data.size, ptrs, _p(lens), 4, C.byref(out), C.byref(n))
    elif enc.codec == "lzss_contig":
        cont = enc.params["container"]
        rc = L.gd_lzss_contig_decompress(_p(cont), cont.size, C.byref(out), C.byref(n))
    elif enc.codec in ("brle_trans", "brle_trans4"):
        fn = L.gd_brle_trans_decompress if enc.codec == "brle_trans" else L.gd_brle_trans4_decompress
        rc = fn(_p(enc.data), enc.data.size, _p(m["col_len"]), m["col_len"].nbytes, _p(m["col_map"]),
                m["col_map"].nbytes, _p(m["blk_off"]), m["blk_off"].nbytes, enc.chunk_size, C.byref(out), C.byref(n))
    elif enc.codec == "deflate":
        oo = m["out_off"]
        cs = int(oo[1] - oo[0]) if enc.n_chunks > 0 else 1
        uniform = enc.n_chunks > 0 and bool((np.diff(oo[:-1].astype(np.int64)) == cs).all()) and \
            0 < int(oo[-1] - oo[-2]) <= cs and enc.params["zlib_header"] == 1
        if uniform:
            # reference triple: blk_offset = [total][0][cumulative], col_len = padded lengths
            blk = np.concatenate([np.array([enc.n_out], dtype=np.uint64), m["comp_off"]])
            rc = L.gd_deflate_decompress(_p(enc.data), enc.data.size, _p(m["comp_len"]), m["comp_len"].nbytes,
                                         _p(blk), blk.nbytes, cs, C.byref(out), C.byref(n))
        else:  # chunks of any size: the extension call with per-chunk output offsets
            rc = L.gd_inflate_decompress(_p(enc.data), enc.data.size, _p(m["comp_off"]), _p(m["comp_len"]),
                                         _p(oo), enc.n_chunks, enc.params["zlib_header"], C.byref(out), C.byref(n))
    else:
        raise ValueError(enc.codec)
    check(rc, f"{enc.codec} host decompress")
    res = None
    if keep:
        res = np.ctypeslib.as_array(C.cast(out, C.POINTER(C.c_uint8)), shape=(n.value,)).copy() if n.value else \
            np.empty(0, np.uint8)
    L.gd_free(out)
    return res
