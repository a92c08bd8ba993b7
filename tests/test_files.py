"""The reference's on-disk layouts (compression_b200.files): every writer's
files have the reference's structure, and every reader gives back a
container the oracle decodes to the column.  CPU only, except the cuDF
reader's flow, which runs on gd_gpuinflate."""
import zlib

import numpy as np
import pytest

import compression_b200.codecs as cc
import compression_b200.files as F
import oracle


def _decodes(enc, raw):
    rc, out = oracle.decode(enc)
    assert rc == 0
    assert np.array_equal(out[:raw.size], raw) and not out[raw.size:].any()


def test_brle_file(tmp_path):
    raw = cc.gen_brle_bytes(1, 3 * 256 * 1024 + 11)
    enc = cc.brle_encode(raw)
    F.write_brle(enc, tmp_path / "c.bin")
    back = F.read_brle(tmp_path / "c.bin")
    assert np.array_equal(back.params["container"], enc.params["container"])
    _decodes(back, raw)


def test_lzss_file_and_meta_sidecar(tmp_path):
    raw = cc.gen_markov_copy(2, 5 * 65536, 4096)
    enc = cc.lzss_encode(raw, 65536)
    F.write_lzss(enc, tmp_path / "l.bin")
    m = np.fromfile(tmp_path / "l.bin.meta", dtype=np.uint8)
    n = enc.n_chunks
    assert int(m[:8].view(np.uint64)[0]) == 4
    assert list(m[8:40].view(np.uint64)) == [8, 8 * (n + 1), 8 * 32 * n, 32 * n]
    assert int(m[40:48].view(np.uint64)[0]) == 65536
    back = F.read_lzss(tmp_path / "l.bin")
    assert np.array_equal(back.data, enc.data) and np.array_equal(back.meta["col_map"], enc.meta["col_map"])
    _decodes(back, raw)


def test_rlev1_file_and_side_files(tmp_path):
    v = cc.gen_rlev1_ints(3, 3 * 32768)
    enc = cc.rlev1_encode(v, 128 * 1024, 128, 4)
    F.write_rlev1(enc, tmp_path / "r.bin", tmp_path / "input_data")
    assert int(np.fromfile(tmp_path / "r.bin", dtype=np.uint64, count=1)[0]) == v.nbytes
    assert (tmp_path / "input_data" / "rle_v1_col_len.bin").stat().st_size == 8 * 32 * enc.n_chunks
    assert (tmp_path / "input_data" / "rle_v1_blk_offset.bin").stat().st_size == 8 * (enc.n_chunks + 1)
    back = F.read_rlev1(tmp_path / "r.bin", tmp_path / "input_data", 128 * 1024, 128, 4)
    _decodes(back, v.view(np.uint8))


@pytest.mark.parametrize("sym,chunk", [(1, 4096), (4, 8192)])
def test_flag_rle_files(tmp_path, sym, chunk):
    raw = cc.gen_brle_bytes(4, 40 * chunk)
    enc = cc.brle_trans_encode(raw, chunk) if sym == 1 else cc.brle_trans4_encode(raw, chunk)
    F.write_brle_trans(enc, tmp_path / "t.bin", tmp_path / "input_data")
    back = F.read_brle_trans(tmp_path / "t.bin", tmp_path / "input_data", chunk, sym)
    assert back.codec == enc.codec
    _decodes(back, raw)


def test_deflate_triple(tmp_path):
    raw = cc.gen_markov_copy(5, 7 * 131072 + 999, 32768)
    cs = 131072
    oo = np.minimum(np.arange(9, dtype=np.uint64) * cs, raw.size).astype(np.uint64)
    enc = cc.deflate_encode(raw, oo, 9)
    F.write_deflate_triple(enc, tmp_path / "d")
    blk = np.fromfile(str(tmp_path / "d") + "_blk_offset.bin", dtype=np.uint64)
    lens = np.fromfile(str(tmp_path / "d") + "_col_len.bin", dtype=np.uint64)
    assert blk[0] == raw.size and blk[1] == 0 and blk.size == 8 + 2            # num_blk = bytes/8 - 2
    assert (lens % 8 == 0).all() and np.array_equal(np.cumsum(lens), blk[2:])  # padded to 8 bytes
    back = F.read_deflate_triple(tmp_path / "d", cs)
    _decodes(back, raw)


def _cudf_file(tmp_path, raw, cs):
    F.write_cudf_single(raw, tmp_path / "c.bin", cs)
    h = np.fromfile(tmp_path / "c.bin", dtype=np.uint64, count=2)
    n = int(h[1])
    assert int(h[0]) == cs and n == (raw.size + cs - 1) // cs
    lens = np.fromfile(tmp_path / "c.bin", dtype=np.uint64, count=n, offset=16)
    data = np.fromfile(tmp_path / "c.bin", dtype=np.uint8, offset=16 + 8 * n)
    assert data.size == lens.sum()
    return n


def test_cudf_single_file(tmp_path):
    raw = cc.gen_markov_copy(6, 5 * 65536 + 123, 32768)
    cs = 65536
    n = _cudf_file(tmp_path, raw, cs)
    # the last chunk is zero-padded before compressing, so the file decodes to whole chunks
    back = F.read_cudf_single(tmp_path / "c.bin", n * cs)
    _decodes(back, raw)
    # each stream is zlib level 9 of its padded chunk, unpadded
    data = np.fromfile(tmp_path / "c.bin", dtype=np.uint8, offset=16 + 8 * n)
    padded = np.zeros(n * cs, np.uint8)
    padded[:raw.size] = raw
    z0 = zlib.compress(padded[:cs].tobytes(), 9)
    assert data[:len(z0)].tobytes() == z0


@pytest.mark.gpu
def test_cudf_single_file_gpu_flow(tmp_path, cuda):
    raw = cc.gen_markov_copy(7, 9 * 65536 + 7, 32768)
    n = _cudf_file(tmp_path, raw, 65536)
    out = F.decode_cudf_single(tmp_path / "c.bin", cuda)
    assert out.size == n * 65536
    assert np.array_equal(out[:raw.size], raw) and not out[raw.size:].any()
