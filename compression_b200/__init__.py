"""compression_b200 -- B200-native (sm_100a) decode library for the
ZaidQureshi/compression containers: byte-RLE, RLE v1, RLE v2, LZSS and
Deflate/zlib, plus a batched mixed-codec decoder.

The decoders are CUDA kernels in libgd.so behind the C ABI in include/gd.h;
this package binds that ABI (``_lib``), mirrors the reference's host
interface (``codecs``), and builds the library (``build``).
"""
from ._lib import lib, LIB_PATH  # noqa: F401

__all__ = ["lib", "LIB_PATH"]
