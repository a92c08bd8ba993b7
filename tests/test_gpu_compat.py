"""A reference-style C++ caller, compiled against include/gd_compat.hpp and
run on the GPU: each codec's compress call followed by its decompress call,
through the reference's own signatures, side files and output ownership.
The compressed bytes equal the host encoders' and the decompressed bytes
equal the column (RLE v2: what the oracle decodes from the same stream)."""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import compression_b200.codecs as cc
import oracle
from compression_b200 import _lib

pytestmark = pytest.mark.gpu

CALLER = r'''
#include "gd_compat.hpp"
#include <iterator>

static std::vector<uint8_t> slurp(const char* p) {
    std::ifstream f(p, std::ios::binary);
    return std::vector<uint8_t>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}
static void dump(const char* p, const void* d, uint64_t n) {
    std::ofstream f(p, std::ios::binary);
    f.write(static_cast<const char*>(d), (std::streamsize)n);
}

int main() {
    uint8_t *c = nullptr, *d = nullptr;
    uint64_t cn = 0, dn = 0;

    std::vector<uint8_t> a = slurp("brle.raw");
    brle::compress_gpu(a.data(), &c, a.size(), &cn);
    if (!c) return 1;
    dump("brle.comp", c, cn);
    brle::decompress_gpu(c, &d, cn, &dn);
    if (!d) return 2;
    dump("brle.out", d, dn);
    delete[] c;
    delete[] d;

    std::vector<uint8_t> b = slurp("rlev1.raw");
    rle_v1::compress_gpu<uint64_t, uint32_t, uint32_t>(b.data(), &c, b.size(), &cn, 128, 128 * 1024);
    if (!c) return 3;
    dump("rlev1.comp", c, cn);
    rle_v1::decompress_gpu<uint64_t, uint32_t, uint32_t, 8>(c, &d, cn, &dn, 128, 128 * 1024);
    if (!d) return 4;
    dump("rlev1.out", d, dn);
    delete[] c;
    delete[] d;

    std::vector<uint8_t> v = slurp("rlev2.raw");
    std::vector<uint64_t> w(v.size() / 8);
    std::memcpy(w.data(), v.data(), w.size() * 8);
    uint8_t* e = nullptr;
    uint64_t en = 0, ms = 0, nch = 0, *bo = nullptr, *cl = nullptr;
    rlev2::compress_gpu_transpose<32, uint64_t>(w.data(), w.size() * 8, e, en, ms, nch, bo, cl, 256 * 1024);
    if (!e || ms != 8 * 32 * nch + 8 * (nch + 1)) return 5;
    dump("rlev2.comp", e, en);
    dump("rlev2.blk", bo, 8 * (nch + 1));
    uint64_t* o64 = nullptr;
    uint64_t on = 0;
    rlev2::decompress_gpu<32, 4, uint64_t>(e, en, nch, bo, cl, o64, on, 256 * 1024);
    if (!o64) return 6;
    dump("rlev2.out", o64, on);
    delete[] e;
    delete[] bo;
    delete[] cl;
    delete[] o64;

    std::vector<uint8_t> z = slurp("lzss.raw");
    uint8_t** meta = nullptr;
    uint64_t* ml = nullptr;
    uint64_t mn = 0;
    lzss::compress_gpu(z.data(), z.size(), &c, &cn, &meta, &ml, &mn);
    if (!c || mn != 4) return 7;
    dump("lzss.comp", c, cn);
    dump("lzss.map", meta[3], ml[3]);
    if (lzss::decompress_gpu(c, cn, (const uint8_t**)meta, ml, mn, &d, &dn) != 0) return 8;
    dump("lzss.out", d, dn);
    for (uint64_t i = 0; i < mn; ++i) free(meta[i]);
    free(meta);
    free(ml);
    delete[] c;
    delete[] d;
    return 0;
}
'''


def _read(p: Path, dtype=np.uint8) -> np.ndarray:
    return np.fromfile(p, dtype=dtype)


def test_reference_style_caller_round_trips(cuda, tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    root = Path(_lib.__file__).resolve().parent.parent
    lib_dir = root / "compression_b200"
    (tmp_path / "caller.cpp").write_text(CALLER)
    exe = tmp_path / "caller"
    r = subprocess.run([gxx, "-std=c++17", "-O1", f"-I{root / 'include'}", str(tmp_path / "caller.cpp"),
                        f"-L{lib_dir}", "-lgd", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr

    raw = {"brle": cc.gen_brle_bytes(3, 1_000_003),
           "rlev1": cc.gen_rlev1_ints(4, 300_000).astype(np.uint32).view(np.uint8),
           "rlev2": cc.gen_rlev2_ints(5, 300_000).view(np.uint8),
           "lzss": cc.gen_markov_copy(6, 3 * 128 * 1024 + 5000, 4096)}
    for k, v in raw.items():
        v.tofile(tmp_path / f"{k}.raw")
    (tmp_path / "input_data").mkdir()   # where rle_v1's side files go
    r = subprocess.run([str(exe)], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stderr)

    host = cc.brle_encode(raw["brle"])
    assert np.array_equal(_read(tmp_path / "brle.comp"), host.params["container"])
    assert np.array_equal(_read(tmp_path / "brle.out"), raw["brle"])

    host = cc.rlev1_encode(raw["rlev1"], 128 * 1024, 128, 4)
    comp = _read(tmp_path / "rlev1.comp")
    assert int(comp[:8].view(np.uint64)[0]) == raw["rlev1"].size
    assert np.array_equal(comp[8:], host.data)
    assert np.array_equal(_read(tmp_path / "input_data" / "rle_v1_col_len.bin", np.uint64), host.meta["col_len"])
    assert np.array_equal(_read(tmp_path / "input_data" / "rle_v1_blk_offset.bin", np.uint64), host.meta["blk_off"])
    assert np.array_equal(_read(tmp_path / "rlev1.out"), raw["rlev1"])

    host = cc.rlev2_encode(raw["rlev2"], 256 * 1024, 32)
    assert np.array_equal(_read(tmp_path / "rlev2.comp"), host.data)
    blk = _read(tmp_path / "rlev2.blk", np.uint64)
    assert np.array_equal(blk[:-1], host.meta["blk_off"][:-1]) and int(blk[-1]) == raw["rlev2"].size
    rc, ref = oracle.decode(host)
    assert rc == 0
    assert np.array_equal(_read(tmp_path / "rlev2.out"), ref)

    host = cc.lzss_encode(raw["lzss"], 128 * 1024)
    assert np.array_equal(_read(tmp_path / "lzss.comp"), host.data)
    assert np.array_equal(_read(tmp_path / "lzss.map"), host.meta["col_map"])
    out = _read(tmp_path / "lzss.out")
    assert out.size == 4 * 128 * 1024 and np.array_equal(out[:raw["lzss"].size], raw["lzss"])
