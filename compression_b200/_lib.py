"""ctypes binding of libgd.so (the C ABI declared in include/gd.h).

The library must have been built in-tree (``python -m compression_b200.build``
or ``__graft_entry__.build()``).  There is no fallback: if the shared object is
missing or fails to load, :func:`lib` raises, and every decode path with it.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libgd.so"

u8p = C.POINTER(C.c_uint8)
u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)
i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)
vp = C.c_void_p
u32 = C.c_uint32
u64 = C.c_uint64
i32 = C.c_int

# name: (restype, argtypes).  Device pointers and streams are passed as void*.
SIGNATURES = {
    "gd_version": (C.c_char_p, []),
    "gd_status_string": (C.c_char_p, [i32]),
    "gd_brle_decode": (i32, [vp, vp, u32, u64, vp, u64, vp, vp]),
    "gd_rlev1_decode": (i32, [vp, vp, vp, u32, u64, u32, u32, vp, u64, u32, vp, vp]),
    "gd_rlev2_decode": (i32, [vp, vp, vp, u32, u64, u32, vp, u64, u32, vp, vp]),
    "gd_lzss_decode": (i32, [vp, vp, vp, vp, u32, u64, vp, u64, vp, vp]),
    "gd_inflate": (i32, [vp, vp, vp, vp, u32, i32, vp, vp, vp]),
    "gd_inflate_ordered": (i32, [vp, vp, vp, vp, u32, i32, vp, vp, vp, vp]),
    "gd_gpuinflate": (i32, [vp, vp, i32, i32, vp]),
    "gd_lzss_contig_decode": (i32, [vp, vp, u32, u64, vp, u64, vp, vp]),
    "gd_brle_trans_decode": (i32, [vp, vp, vp, vp, u32, u64, vp, u64, vp, vp]),
    "gd_brle_trans4_decode": (i32, [vp, vp, vp, vp, u32, u64, vp, u64, vp, vp]),
    "gd_copy_uncompressed_blocks": (i32, [vp, i32, vp]),
    "gd_batch_decode": (i32, [vp, u32, vp, i32, u32, u32, vp, vp, vp, vp]),
    "gd_batch_warps": (u32, [u32, u32]),
    "gd_batch_decode_lpt_noalloc": (i32, [vp, u32, vp, u32, u32, vp, vp]),
    "gd_tune_set": (i32, [i32, i32]),
    "gd_tune_get": (i32, [i32]),
    "gd_mlp_num_params": (u32, []),
    "gd_mlp_predict": (i32, [vp, vp, u32, vp, vp]),
    "gd_mlp_train_step": (i32, [vp, vp, vp, vp, vp, vp, u32, C.c_float, C.c_float, C.c_float, C.c_float, u32, vp,
                                vp, vp]),
    "gd_free": (None, [vp]),
    "gd_brle_decompress": (i32, [vp, u64, C.POINTER(vp), u64p]),
    "gd_rlev1_decompress": (i32, [vp, u64, vp, u64, vp, u64, u32, u32, u64, C.POINTER(vp), u64p]),
    "gd_rlev2_decompress": (i32, [vp, u64, u64, vp, vp, u32, u64, C.POINTER(vp), u64p]),
    "gd_lzss_decompress": (i32, [vp, u64, vp, vp, u64, C.POINTER(vp), u64p]),
    "gd_deflate_decompress": (i32, [vp, u64, vp, u64, vp, u64, u64, C.POINTER(vp), u64p]),
    "gd_lzss_contig_decompress": (i32, [vp, u64, vp, vp]),
    "gd_inflate_decompress": (i32, [vp, u64, vp, vp, vp, u32, i32, vp, vp]),
    "gd_brle_trans_decompress": (i32, [vp, u64, vp, u64, vp, u64, vp, u64, u64, vp, vp]),
    "gd_brle_trans4_decompress": (i32, [vp, u64, vp, u64, vp, u64, vp, u64, u64, vp, vp]),
    "gd_brle_max_encoded_bytes": (u64, [u64, u64]),
    "gd_brle_encode": (u64, [vp, u64, u64, vp]),
    "gd_rlev1_max_encoded_bytes": (u64, [u64, u64]),
    "gd_rlev1_encode": (u64, [vp, u64, u64, u32, u32, vp, vp, vp]),
    "gd_rlev1_encode_stream": (u64, [vp, u64, u32, vp, u64]),
    "gd_rlev2_max_encoded_bytes": (u64, [u64, u64]),
    "gd_rlev2_encode": (u64, [vp, u64, u64, u32, vp, vp, vp]),
    "gd_rlev2_encode_stream": (u64, [vp, u64, vp, u64]),
    "gd_brle_encode_scratch_bytes": (u64, [u64, u64]),
    "gd_brle_encode_device": (i32, [vp, u64, u64, vp, vp, vp, vp]),
    "gd_lzss_encode_bound": (u64, [u64, u64]),
    "gd_brle_trans_encode_bound": (u64, [u64, u64]),
    "gd_lzss_encode_device": (i32, [vp, u64, u64, vp, vp, vp, vp, vp, vp, vp]),
    "gd_brle_trans_encode_device": (i32, [vp, u64, u64, vp, vp, vp, vp, vp, vp, vp]),
    "gd_rlev1_encode_bound": (u64, [u64, u64, u32]),
    "gd_rlev1_encode_device": (i32, [vp, u64, u64, u32, u32, vp, vp, vp, vp, vp, vp]),
    "gd_rlev2_encode_bound": (u64, [u64, u64]),
    "gd_rlev2_encode_device": (i32, [vp, u64, u64, u32, vp, vp, vp, vp, vp, vp]),
    "gd_brle_compress": (i32, [vp, u64, vp, vp]),
    "gd_rlev1_compress": (i32, [vp, u64, u32, u32, u64, vp, vp, vp, vp, vp]),
    "gd_rlev2_compress": (i32, [vp, u64, u32, u64, vp, vp, vp, vp, vp]),
    "gd_lzss_compress": (i32, [vp, u64, vp, vp, vp, vp, vp]),
    "gd_lzss_max_encoded_bytes": (u64, [u64, u64]),
    "gd_lzss_encode": (u64, [vp, u64, u64, vp, vp, vp, vp]),
    "gd_lzss_encode_stream": (u64, [vp, u32, vp, u64]),
    "gd_lzss_contig_max_encoded_bytes": (u64, [u64, u64]),
    "gd_lzss_contig_encode": (u64, [vp, u64, u64, vp]),
    "gd_brle_trans_max_encoded_bytes": (u64, [u64, u64]),
    "gd_brle_trans_encode": (u64, [vp, u64, u64, vp, vp, vp, vp]),
    "gd_brle_trans4_max_encoded_bytes": (u64, [u64, u64]),
    "gd_brle_trans4_encode": (u64, [vp, u64, u64, vp, vp, vp, vp]),
    "gd_deflate_max_encoded_bytes": (u64, [vp, u32]),
    "gd_deflate_encode": (u64, [vp, vp, u32, i32, vp, i32, vp, vp, vp]),
    "gd_task_features": (i32, [vp, u32, vp, vp]),
    "gd_gen_rlev1_ints": (None, [u64, u64, vp]),
    "gd_gen_brle_bytes": (None, [u64, u64, vp]),
    "gd_gen_rlev2_ints": (None, [u64, u64, vp]),
    "gd_gen_markov_copy": (None, [u64, u64, u32, vp]),
    "gd_gen_loguniform_sizes": (i32, [u64, u32, u64, u64, u64, u64, vp]),
}

_LIB = None


def lib() -> C.CDLL:
    """Load libgd.so once and attach the C signatures."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is not built; run `python -m compression_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


def declared_symbols() -> list[str]:
    """Function names declared in include/gd.h (parsed from the header)."""
    import re
    hdr = (_HERE.parent / "include" / "gd.h").read_text()
    return sorted(set(re.findall(r"\b(gd_[a-z0-9_]+)\s*\(", hdr)))
