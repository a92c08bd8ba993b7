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
    # device encoders: partial values, chunk not a multiple of 32 slices, unaligned input
    assert L.gd_rlev1_encode_device(4, 999, 4096, 128, 4, 4, 4, 8, 8, None, None) == 1
    assert L.gd_rlev1_encode_device(4, 1000, 4000, 128, 4, 4, 4, 8, 8, None, None) == 1
    assert L.gd_rlev1_encode_device(2, 1000, 4096, 128, 4, 4, 4, 8, 8, None, None) == 1
    assert L.gd_rlev2_encode_device(8, 996, 8192, 1, 4, 4, 8, 8, None, None) == 1
    assert L.gd_rlev2_encode_device(8, 1000, 8192, 3, 4, 4, 8, 8, None, None) == 1
    assert L.gd_rlev1_encode_device(None, 0, 4096, 128, 4, None, None, None, None, None, None) == 0  # empty
    assert L.gd_brle_encode_device(None, 100, 4096, 16, 4, 8, None) == 1          # no input
    assert L.gd_brle_encode_device(1, 100, 4096, 8, 4, 8, None) == 1             # scratch not 16-aligned
    assert L.gd_brle_encode_device(1, 0, 4096, 16, 4, 8, None) == 1              # empty column
    assert L.gd_brle_encode_scratch_bytes(0, 4096) == 0
    assert L.gd_lzss_encode_device(4, 1000, 1000, 4, 4, 8, 8, 1, None, None) == 1     # chunk % 128
    assert L.gd_lzss_encode_device(4, 1000, 256 * 1024, 4, 4, 8, 8, 1, None, None) == 1  # column > 4 KiB
    assert L.gd_lzss_encode_device(2, 1000, 4096, 4, 4, 8, 8, 1, None, None) == 1     # unaligned input
    assert L.gd_brle_trans_encode_device(4, 1000, 1000, 4, 4, 8, 8, 1, None, None) == 1   # chunk % 128
    assert L.gd_brle_trans_encode_device(4, 1000, 8192, 4, 4, 8, 8, 1, None, None) == 1   # column > 252 bytes
    assert L.gd_brle_trans_encode_device(2, 1000, 4096, 4, 4, 8, 8, 1, None, None) == 1   # unaligned input
    assert L.gd_brle_trans_encode_device(4, 1000, 4096, 4, None, 8, 8, 1, None, None) == 1  # no data buffer
    assert L.gd_brle_trans_encode_bound(2 * 4096, 4096) == 2 * 32 * (((128 + 16 + 8 + 3) & ~3) + 4) + 16
    # bounds: 32 lane slots per chunk, each holding the longest lane stream
    assert L.gd_rlev1_encode_bound(128 * 1024, 128 * 1024, 4) == 32 * ((1024 * 5 + 1024 // 64 + 16 + 3) & ~3)
    assert L.gd_rlev2_encode_bound(2 * 256 * 1024, 256 * 1024) == 2 * 32 * ((1024 * 11 + 64 + 3) & ~3)


def test_compat_header_compiles_and_links(tmp_path):
    # a reference-style caller: the reference's namespaced calls from
    # include/gd_compat.hpp, linked against libgd.so (compiled, not run)
    import shutil
    import subprocess
    from pathlib import Path
    gxx = shutil.which("g++")
    if gxx is None:
        import pytest
        pytest.skip("no g++")
    root = Path(_lib.__file__).resolve().parent.parent
    src = tmp_path / "caller.cpp"
    src.write_text(r'''
#include "gd_compat.hpp"
int main(int argc, char**) {
    uint8_t* out = nullptr; uint64_t n = 0;
    if (argc > 5) {
        brle::decompress_gpu(nullptr, &out, 0, &n);
        rle_v1::decompress_gpu<uint64_t, uint8_t, uint32_t, 2>(nullptr, &out, 0, &n, 128, 128 * 1024);
        uint64_t* o64 = nullptr; uint64_t bo[2] = {0, 0}, cl[32] = {};
        rlev2::decompress_gpu<32, 4, uint64_t>(nullptr, 0, 1, bo, cl, o64, n, 256 * 1024);
        lzss::decompress_gpu(nullptr, 0, nullptr, nullptr, 4, &out, &n);
        lzss::decompress_gpu_base(nullptr, &out, 0, &n);
        brle_trans::decompress_gpu(nullptr, &out, 0, &n);
        deflate::decompress_gpu<uint64_t, 8, 2, 1>(nullptr, &out, 0, &n, cl, 8, bo, 16, 65536);
        cudf::io::gpuinflate(nullptr, nullptr, 0, 1);
        brle::compress_gpu(nullptr, &out, 0, &n);
        rle_v1::compress_gpu<uint64_t, uint32_t, uint32_t>(nullptr, &out, 0, &n, 128, 128 * 1024);
        uint8_t* enc = nullptr; uint64_t ms = 0, nch = 0; uint64_t* pbo = nullptr; uint64_t* pcl = nullptr;
        const uint64_t* in64 = nullptr;
        rlev2::compress_gpu_transpose<32, uint64_t>(in64, 0, enc, n, ms, nch, pbo, pcl, 256 * 1024);
        uint8_t** meta = nullptr; uint64_t* ml = nullptr; uint64_t mn = 0;
        lzss::compress_gpu(nullptr, 0, &out, &n, &meta, &ml, &mn);
    }
    return 0;
}
''')
    exe = tmp_path / "caller"
    lib_dir = root / "compression_b200"
    r = subprocess.run([gxx, "-std=c++17", f"-I{root / 'include'}", str(src), f"-L{lib_dir}", "-lgd",
                        f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert subprocess.run([str(exe)]).returncode == 0


def test_tuning_knobs_set_and_get():
    L = _lib.lib()
    n_keys = 7  # GD_TUNE_COUNT
    for key in range(n_keys):
        old = L.gd_tune_get(key)
        assert old >= 0
        assert L.gd_tune_set(key, 4) == old
        assert L.gd_tune_get(key) == 4
        assert L.gd_tune_set(key, old) == 4
    assert L.gd_tune_get(n_keys) == -1 and L.gd_tune_set(n_keys, 1) == -1 and L.gd_tune_set(0, -1) == -1


def test_host_compress_argument_errors():
    # rejected on the host, before any device call
    import ctypes as C
    L = _lib.lib()
    out, n, a, b, k = C.c_void_p(), C.c_uint64(), C.c_void_p(), C.c_void_p(), C.c_uint64()
    buf = (C.c_uint8 * 16)()
    bad = [L.gd_brle_compress(None, 16, C.byref(out), C.byref(n)),
           L.gd_brle_compress(buf, 0, C.byref(out), C.byref(n)),
           L.gd_rlev1_compress(buf, 0, 128, 4, 4096, C.byref(out), C.byref(n), C.byref(a), C.byref(b), C.byref(k)),
           L.gd_rlev1_compress(buf, 16, 128, 4, 0, C.byref(out), C.byref(n), C.byref(a), C.byref(b), C.byref(k)),
           L.gd_rlev2_compress(buf, 0, 32, 8192, C.byref(out), C.byref(n), C.byref(a), C.byref(b), C.byref(k)),
           L.gd_rlev2_compress(buf, 16, 32, 8192, None, C.byref(n), C.byref(a), C.byref(b), C.byref(k)),
           L.gd_lzss_compress(buf, 0, C.byref(out), C.byref(n), C.byref(a), C.byref(b), C.byref(k)),
           L.gd_lzss_compress(buf, 16, C.byref(out), C.byref(n), None, C.byref(b), C.byref(k))]
    assert all(L.gd_status_string(rc) == b"invalid argument" for rc in bad), bad
