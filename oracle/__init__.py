"""CPU oracle for the decode hot path -- TEST INFRASTRUCTURE ONLY.

A plain-C restatement of the reference decoders (gd_oracle.c, built into
liboracle.so by oracle/build.py) plus system zlib for Deflate.  Only tests/,
__graft_entry__.smoke() and the CPU-baseline leg of bench.py use it, as the
checker; the compression_b200 package never imports it.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
_L = None

vp, u32, u64, i32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int


def lib():
    global _L
    if _L is None:
        if not LIB_PATH.exists():
            from . import build as _b  # noqa: F401  (oracle/build.py)
            _b.build_oracle()
        L = C.CDLL(str(LIB_PATH))
        L.gdo_brle_decode.argtypes = [vp, vp, u32, u64, vp, u64]
        L.gdo_rlev1_decode.argtypes = [vp, u64, vp, vp, u32, u64, u32, u32, vp, u64]
        L.gdo_rlev2_decode.argtypes = [vp, u64, vp, vp, u32, u64, u32, vp, u64]
        L.gdo_lzss_decode.argtypes = [vp, u64, vp, vp, vp, u32, u64, vp, u64]
        L.gdo_inflate.argtypes = [vp, vp, vp, vp, u32, i32, vp]
        L.gdo_lzss_contig_decode.argtypes = [vp, u64, vp, u64]
        L.gdo_brle_trans_decode.argtypes = [vp, u64, vp, vp, vp, u32, u64, vp, u64]
        L.gdo_brle_trans4_decode.argtypes = [vp, u64, vp, vp, vp, u32, u64, vp, u64]
        for f in ("gdo_brle_decode", "gdo_rlev1_decode", "gdo_rlev2_decode", "gdo_lzss_decode", "gdo_inflate",
                  "gdo_lzss_contig_decode", "gdo_brle_trans_decode", "gdo_brle_trans4_decode"):
            getattr(L, f).restype = i32
        L.gdo_rlev2_decode_stream.argtypes = [vp, u64, vp, u64]
        L.gdo_lzss_decode_stream.argtypes = [vp, u64, vp, u64]
        L.gdo_rlev2_decode_stream.restype = i32
        L.gdo_lzss_decode_stream.restype = i32
        L.gdo_export_lanes.argtypes = [vp, u64, vp, vp, u32, vp, vp]
        L.gdo_export_lanes.restype = i32
        L.gdo_version.restype = C.c_char_p
        L.gdo_rlev1_encode.argtypes = [vp, u64, u64, u32, u32, vp, vp, vp]
        L.gdo_rlev1_encode.restype = u64
        L.gdo_rlev1_max_encoded_bytes.argtypes = [u64, u64]
        L.gdo_rlev1_max_encoded_bytes.restype = u64
        for f in ("gd_gen_rlev1_ints", "gd_gen_brle_bytes", "gd_gen_rlev2_ints"):
            getattr(L, f).argtypes = [u64, u64, vp]
            getattr(L, f).restype = None
        L.gd_gen_markov_copy.argtypes = [u64, u64, u32, vp]
        L.gd_gen_markov_copy.restype = None
        L.gd_gen_loguniform_sizes.argtypes = [u64, u32, u64, u64, u64, u64, vp]
        L.gd_gen_loguniform_sizes.restype = i32
        _L = L
    return _L


def _p(a):
    return a.ctypes.data


def decode(enc) -> tuple[int, np.ndarray]:
    """Decode a compression_b200.codecs.Encoded container on the CPU.

    Returns (status, output bytes)."""
    L = lib()
    m = enc.meta
    out = np.zeros(max(enc.n_out, 1), dtype=np.uint8)
    d = enc.data
    if enc.codec == "brle":
        rc = L.gdo_brle_decode(_p(d), _p(m["ptr"]), enc.n_chunks, enc.chunk_size, _p(out), enc.n_out)
    elif enc.codec == "rlev1":
        rc = L.gdo_rlev1_decode(_p(d), d.size, _p(m["blk_off"]), _p(m["col_len"]), enc.n_chunks, enc.chunk_size,
                                enc.params["comp_col_len"], enc.params["elem_bytes"], _p(out), enc.n_out)
    elif enc.codec == "rlev2":
        rc = L.gdo_rlev2_decode(_p(d), d.size, _p(m["blk_off"]), _p(m["col_len"]), enc.n_chunks, enc.chunk_size,
                                enc.params["read_unit"], _p(out), enc.n_out)
    elif enc.codec == "lzss":
        rc = L.gdo_lzss_decode(_p(d), d.size, _p(m["blk_off"]), _p(m["col_len"]), _p(m["col_map"]),
                               enc.n_chunks, enc.chunk_size, _p(out), enc.n_out)
    elif enc.codec == "lzss_contig":
        cont = enc.params["container"]
        rc = L.gdo_lzss_contig_decode(_p(cont), cont.size, _p(out), out.size)
    elif enc.codec == "brle_trans":
        rc = L.gdo_brle_trans_decode(_p(d), d.size, _p(m["blk_off"]), _p(m["col_len"]), _p(m["col_map"]),
                                     enc.n_chunks, enc.chunk_size, _p(out), enc.n_out)
    elif enc.codec == "brle_trans4":
        rc = L.gdo_brle_trans4_decode(_p(d), d.size, _p(m["blk_off"]), _p(m["col_len"]), _p(m["col_map"]),
                                      enc.n_chunks, enc.chunk_size, _p(out), enc.n_out)
    elif enc.codec == "deflate":
        rc = L.gdo_inflate(_p(d), _p(m["comp_off"]), _p(m["comp_len"]), _p(m["out_off"]), enc.n_chunks,
                           enc.params["zlib_header"], _p(out))
    else:
        raise ValueError(enc.codec)
    return int(rc), out[: enc.n_out]


def rlev2_decode_stream(stream: np.ndarray, n_vals: int) -> tuple[int, np.ndarray]:
    s = np.ascontiguousarray(stream, dtype=np.uint8)
    out = np.zeros(n_vals, dtype=np.int64)
    return int(lib().gdo_rlev2_decode_stream(_p(s), s.size, _p(out), n_vals)), out


def lzss_decode_stream(stream: np.ndarray, n_out: int) -> tuple[int, np.ndarray]:
    s = np.ascontiguousarray(stream, dtype=np.uint8)
    out = np.zeros(n_out, dtype=np.uint8)
    return int(lib().gdo_lzss_decode_stream(_p(s), s.size, _p(out), n_out)), out


def export_lanes(enc) -> tuple[np.ndarray, np.ndarray]:
    """The 32 * n_chunks lane (or column) streams of an interleaved container
    back to back, in slot order, and their offsets (32 * n_chunks + 1)."""
    m = enc.meta
    cl = np.ascontiguousarray(m["col_len"], dtype=np.uint64)
    out = np.zeros(max(int(cl.sum()), 1), dtype=np.uint8)
    off = np.zeros(cl.size + 1, dtype=np.uint64)
    rc = lib().gdo_export_lanes(_p(enc.data), enc.data.size, _p(m["blk_off"]), _p(cl), enc.n_chunks,
                                _p(out), _p(off))
    if rc:
        raise RuntimeError(f"export_lanes: status {rc}")
    return out[: int(off[-1])], off


# --------------------------------------------------------------------------
# input builders for the CPU baselines (the reference arm of bench.py builds
# its inputs without the product library)
# --------------------------------------------------------------------------

class Container:
    """A compressed column in the shape decode() reads: codec, payload, meta
    arrays, parameters (the fields of compression_b200.codecs.Encoded)."""

    def __init__(self, codec, data, n_out, n_chunks, chunk_size=0, meta=None, params=None):
        self.codec, self.data, self.n_out, self.n_chunks = codec, data, int(n_out), int(n_chunks)
        self.chunk_size, self.meta, self.params = int(chunk_size), meta or {}, params or {}

    @property
    def comp_bytes(self) -> int:
        return int(self.data.nbytes)

    @property
    def meta_bytes(self) -> int:
        return int(sum(v.nbytes for v in self.meta.values()))


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
    if lib().gd_gen_loguniform_sizes(seed, n, lo, hi, total, granule, _p(a)) != 0:
        raise ValueError("loguniform_sizes")
    return a


def rlev1_encode(raw, chunk_size: int = 128 * 1024, comp_col_len: int = 128, elem_bytes: int = 4) -> Container:
    """The RLE v1 container of `raw` (gd_inputs.cpp)."""
    b = np.ascontiguousarray(raw).view(np.uint8).reshape(-1)
    L = lib()
    nc = (b.size + chunk_size - 1) // chunk_size
    data = np.empty(L.gdo_rlev1_max_encoded_bytes(b.size, chunk_size), dtype=np.uint8)
    blk = np.empty(nc + 1, dtype=np.uint64)
    col = np.empty(32 * nc, dtype=np.uint64)
    n = L.gdo_rlev1_encode(_p(b), b.size, chunk_size, comp_col_len, elem_bytes, _p(data), _p(blk), _p(col))
    if n == 0:
        raise ValueError("rlev1 encode failed")
    return Container("rlev1", data[:n].copy(), b.size, nc, chunk_size, {"blk_off": blk, "col_len": col},
                     {"comp_col_len": comp_col_len, "elem_bytes": elem_bytes})
