"""The C ABI library loads and exports every entry point include/gd.h declares
(no GPU needed: nothing here launches a kernel)."""
import ctypes

from compression_b200 import _lib


def test_library_loads_and_versions():
    L = _lib.lib()
    assert b"sm_100a" in L.gd_version()
    assert L.gd_status_string(2) == b"corrupt stream"


def test_every_declared_symbol_is_exported():
    L = ctypes.CDLL(str(_lib.LIB_PATH))
    declared = _lib.declared_symbols()
    assert len(declared) > 20
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing


def test_bindings_cover_header():
    declared = set(_lib.declared_symbols())
    bound = set(_lib.SIGNATURES)
    assert declared <= bound, sorted(declared - bound)


def test_device_api_rejects_bad_arguments_without_gpu():
    # argument validation happens before any CUDA call
    L = _lib.lib()
    assert L.gd_brle_decode(None, None, 1, 256 * 1024, None, 10, None, None) == 1
    assert L.gd_rlev1_decode(1, 1, 1, 1, 1000, 128, 4, 1, 1000, 0, None, None) == 1  # chunk % (32*128)
    assert L.gd_rlev2_decode(1, 1, 1, 1, 256 * 1024, 0, 1, 10, 0, None, None) == 5
    assert L.gd_lzss_decode(1, 1, 1, 1, 2, 65536, 16, 1000, None, None) == 1  # out != n*chunk
    assert L.gd_inflate(3, 1, 1, 1, 1, 1, 1, None, None) == 1  # unaligned data
