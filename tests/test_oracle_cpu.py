"""CPU-side tests: encoders + oracle round trips, edge cases, corrupt inputs.

The oracle (oracle/gd_oracle.c) is the checker for the GPU tests; here it is
checked against the original input (every container round-trips) and, in
test_golden.py, against outputs of the reference's own code."""
import numpy as np
import pytest

import compression_b200.codecs as cc
import oracle


def _roundtrip(enc, raw_bytes):
    rc, out = oracle.decode(enc)
    assert rc == 0
    assert np.array_equal(out, raw_bytes)


@pytest.mark.parametrize("n", [1, 2, 3, 129, 130, 131, 256 * 1024, 256 * 1024 + 7, 3 * 256 * 1024])
def test_brle_roundtrip_sizes(n):
    raw = cc.gen_brle_bytes(n, n)
    _roundtrip(cc.brle_encode(raw), raw)


def test_brle_patterns():
    rng = np.random.default_rng(0)
    for raw in [np.zeros(5000, np.uint8), np.arange(5000, dtype=np.uint8),
                rng.integers(0, 3, 70000).astype(np.uint8), np.repeat(rng.integers(0, 256, 300), 200).astype(np.uint8)]:
        _roundtrip(cc.brle_encode(raw, 4096), raw)


@pytest.mark.parametrize("eb,ccl", [(4, 128), (4, 16), (8, 64), (4, 256)])
def test_rlev1_roundtrip(eb, ccl):
    v = cc.gen_rlev1_ints(eb + ccl, 70000)
    raw = v.astype(np.int64) if eb == 8 else v
    enc = cc.rlev1_encode(raw, 32 * ccl * 8, ccl, eb)
    rc, out = oracle.decode(enc)
    assert rc == 0 and np.array_equal(out, raw.view(np.uint8))


def test_rlev1_edge_values():
    raw = np.array([0, 0xFFFFFFFF, 5, 5, 5, 7, 9, 11, 13, 1, 2] * 2000, dtype=np.uint32)
    enc = cc.rlev1_encode(raw, 32 * 128, 128, 4)
    _roundtrip(enc, raw.view(np.uint8))


@pytest.mark.parametrize("ru", [1, 4, 32, 64])
def test_rlev2_roundtrip(ru):
    v = cc.gen_rlev2_ints(ru, 40000)
    enc = cc.rlev2_encode(v, 256 * ru * 4, ru)
    _roundtrip(enc, v.view(np.uint8))


def test_rlev2_negative_and_wide_values():
    rng = np.random.default_rng(1)
    v = np.concatenate([rng.integers(-2**62, 2**62, 3000), -np.arange(3000), np.full(500, -7),
                        rng.integers(0, 2**12, 3000) + (rng.random(3000) < 0.03) * 2**50]).astype(np.int64)
    enc = cc.rlev2_encode(v, 256 * 8 * 2, 8)
    _roundtrip(enc, v.view(np.uint8))


@pytest.mark.parametrize("chunk", [128, 4096, 65536])
def test_lzss_roundtrip(chunk):
    raw = cc.gen_markov_copy(chunk, 3 * chunk, 4096)
    _roundtrip(cc.lzss_encode(raw, chunk), raw)


def test_lzss_degenerate():
    for raw in [np.zeros(8192, np.uint8), np.tile(np.arange(7, dtype=np.uint8), 2000)[:8192]]:
        _roundtrip(cc.lzss_encode(raw, 4096), raw)


def test_deflate_modes():
    raw = cc.gen_markov_copy(9, 300000, 32768)
    oo = np.array([0, 1, 4097, 100000, 100000, 300000], dtype=np.uint64)  # includes an empty chunk
    for zh in (0, 1):
        for m in (0, 1, 2):
            enc = cc.deflate_encode(raw, oo, 6, np.full(5, m, np.uint8), zh)
            _roundtrip(enc, raw)


def test_oracle_rejects_corruption():
    raw = cc.gen_brle_bytes(3, 300000)
    enc = cc.brle_encode(raw)
    enc.data[5] = 200  # a literal header claiming bytes that turn into extra output
    rc, _ = oracle.decode(enc)
    assert rc in (2, 3)
    v = cc.gen_rlev2_ints(3, 20000)
    e2 = cc.rlev2_encode(v, 256 * 32, 32)
    e2.meta["col_len"][0] += 4
    rc, _ = oracle.decode(e2)
    assert rc != 0


def test_lzss_partial_last_chunk():
    raw = cc.gen_markov_copy(12, 3 * 65536 + 1000, 4096)
    _roundtrip(cc.lzss_encode(raw, 65536), raw)


def test_mixed_batch_items_roundtrip():
    import compression_b200.batch as B
    items = B.make_mixed_batch(3, 40, 8 << 20)
    assert {it.codec for it in items} == set(B.CODECS)
    for it in items:
        rc, out = oracle.decode(it.enc)
        assert rc == 0 and np.array_equal(out, it.raw), it.codec


@pytest.mark.parametrize("n,chunk", [(1, 1024), (5000, 4096), (3 * 65536, 65536), (300000, 65536)])
def test_lzss_contig_roundtrip(n, chunk):
    raw = cc.gen_markov_copy(n, n, 4096)
    e = cc.lzss_contig_encode(raw, chunk)
    cont = e.params["container"]
    # header: in_n_bytes, chunk_size, n_chunks, history, min and max match (lzss.h:1107-1113)
    assert int(cont[:8].view(np.uint64)[0]) == n
    assert list(cont[8:28].view(np.uint32)) == [chunk, e.n_chunks, 2048, 3, 34]
    _roundtrip(e, raw)


def test_lzss_contig_chunk_streams_are_column_streams():
    # every chunk's stream is the reference grammar's tokenisation of that chunk
    raw = cc.gen_markov_copy(31, 3 * 8192 + 77, 4096)
    e = cc.lzss_contig_encode(raw, 8192)
    L = cc.lib()
    beg = 0
    for c in range(e.n_chunks):
        part = raw[c * 8192:(c + 1) * 8192].copy()
        buf = np.zeros(part.size * 2 + 64, np.uint8)
        n = L.gd_lzss_encode_stream(part.ctypes.data, part.size, buf.ctypes.data, buf.size)
        end = int(e.meta["ends"][c])
        assert np.array_equal(e.data[beg:end], buf[:n])
        beg = end


@pytest.mark.parametrize("n,chunk", [(128, 128), (4096 * 50, 4096), (4096 * 7 + 1000, 4096), (8192 * 3, 8192)])
def test_brle_trans_roundtrip(n, chunk):
    raw = cc.gen_brle_bytes(n + chunk, n)
    _roundtrip(cc.brle_trans_encode(raw, chunk), raw)


def test_brle_trans_patterns():
    rng = np.random.default_rng(4)
    for raw in [np.zeros(4 * 4096, np.uint8), rng.integers(0, 256, 4 * 4096).astype(np.uint8),
                np.repeat(rng.integers(0, 4, 2048), 8).astype(np.uint8)]:
        e = cc.brle_trans_encode(raw, 4096)
        _roundtrip(e, raw)
    # an all-zero column is one run item: flag byte, count 128, value
    e = cc.brle_trans_encode(np.zeros(4096, np.uint8), 4096)
    assert (e.meta["col_len"] == 3).all()
    w = e.data[:128].reshape(32, 4)  # one word row: rank r's word 0 at bytes 4r..4r+3
    assert (w[:, :3] == [0, 128, 0]).all()


def test_brle_trans_column_grammar():
    # column 0 of a chunk: runs of 5 x 7, then 2 x 9 (literals), then 3 x 1
    col = np.array([7] * 5 + [9, 9] + [1] * 3 + [4] * 118, np.uint8)
    raw = np.zeros(4096, np.uint8)
    for k in range(32):
        raw[128 * k:128 * k + 4] = col[4 * k:4 * k + 4]
    e = cc.brle_trans_encode(raw, 4096)
    r = int(np.nonzero(e.meta["col_map"][:32] == 0)[0][0])
    assert int(e.meta["col_len"][r]) == 1 + 2 + 1 + 1 + 2 + 2
    rc, out = oracle.decode(e)
    assert rc == 0 and np.array_equal(out, raw)


def _sym_column_chunk(col: np.ndarray) -> np.ndarray:
    """An 8 KiB chunk whose column 0 holds `col` (256 bytes); the other
    columns are zero."""
    raw = np.zeros(8192, np.uint8)
    for k in range(64):
        raw[128 * k:128 * k + 4] = col[4 * k:4 * k + 4]
    return raw


@pytest.mark.parametrize("n,chunk", [(8192 * 20, 8192), (8192 * 3 + 1000, 8192), (4096 * 9, 4096), (128 * 5, 128)])
def test_brle_trans4_roundtrip(n, chunk):
    rng = np.random.default_rng(n)
    # 4-byte symbols: runs of equal words, as a column of int32 values sees them
    words = np.repeat(rng.integers(0, 6, n // 40 + 1), rng.integers(1, 20, n // 40 + 1)).astype(np.uint32)
    raw = np.resize(words, (n + 3) // 4).view(np.uint8)[:n].copy()
    _roundtrip(cc.brle_trans4_encode(raw, chunk), raw)
    raw = rng.integers(0, 256, n).astype(np.uint8)
    _roundtrip(cc.brle_trans4_encode(raw, chunk), raw)


def test_brle_trans4_column_grammar():
    # column 0 (64 symbols): 5 x A, 2 x B, 56 x C, 1 x D, as the reference's
    # compress_func writes it (brle_gpu_4B.h:321-638): flag byte, run item
    # (count, symbol), literal items (symbol), flag bits LSB first
    A, B, C, D = (np.frombuffer(x, np.uint8) for x in (b"AAAA", b"BBBB", b"CCCC", b"DDDD"))
    col = np.concatenate([A] * 5 + [B] * 2 + [C] * 56 + [D])
    e = cc.brle_trans4_encode(_sym_column_chunk(col), 8192)
    r = int(np.nonzero(e.meta["col_map"][:32] == 0)[0][0])
    n = int(e.meta["col_len"][r])
    lanes, off = oracle.export_lanes(cc.Encoded("lzss", e.data, e.n_out, e.n_chunks, e.chunk_size, e.meta, {}))
    stream = lanes[off[r]:off[r + 1]]
    want = np.concatenate([[0b10110], [5], A, B, B, [56], C, D]).astype(np.uint8)
    assert n == want.size and np.array_equal(stream, want)
    rc, out = oracle.decode(e)
    assert rc == 0 and np.array_equal(out, _sym_column_chunk(col))


def test_brle_trans4_group_ends():
    A = np.frombuffer(b"\x01\x02\x03\x04", np.uint8)
    B = np.frombuffer(b"\x05\x06\x07\x08", np.uint8)
    # 8 literal items end a group: a reserved flag byte follows the last one
    lit = np.concatenate([np.full(4, i, np.uint8) for i in range(1, 9)])
    col = np.concatenate([lit, np.tile(np.concatenate([A, B]), 28)])
    e = cc.brle_trans4_encode(_sym_column_chunk(col), 8192)
    rc, out = oracle.decode(e)
    assert rc == 0 and np.array_equal(out, _sym_column_chunk(col))
    # 7 literal items then a final run: the run closes the group with no
    # reserved flag byte after it (the reference writes the last run uncounted)
    col = np.concatenate([np.concatenate([np.full(4, i, np.uint8) for i in range(1, 8)]), np.tile(A, 57)])
    e = cc.brle_trans4_encode(_sym_column_chunk(col), 8192)
    r = int(np.nonzero(e.meta["col_map"][:32] == 0)[0][0])
    assert int(e.meta["col_len"][r]) == 1 + 7 * 4 + 5
    rc, out = oracle.decode(e)
    assert rc == 0 and np.array_equal(out, _sym_column_chunk(col))


def _ref_compress_func_4B(col: np.ndarray) -> bytes:
    """brle::compress_func of include/brle/brle_gpu_4B.h:321-638 for one
    column, restated loop for loop over an output zeroed beforehand (the
    reference's output buffer is not cleared: a reserved flag byte that no
    item follows keeps whatever was there)."""
    syms = [bytes(col[4 * k:4 * k + 4]) for k in range(col.size // 4)]
    out = bytearray(col.size * 2 + 16)
    pos = 1                    # byte_offset: header byte 0 reserved
    hdr, header, blocks = 0, 0, 0
    counter, prev = 0, None

    def item_done():
        nonlocal blocks, header, hdr, pos
        blocks += 1
        if blocks == 8:
            out[hdr] = header
            header = 0
            hdr = pos
            pos += 1
            blocks = 0
        if blocks != 0:
            out[hdr] = header

    def put(bs):
        nonlocal pos
        out[pos:pos + len(bs)] = bs
        pos += len(bs)

    for v in syms:
        if counter == 0:
            prev = v
        if prev == v:
            counter += 1
            continue
        if counter >= 3:
            put(bytes([counter]) + prev)
            item_done()
        else:
            for _ in range(counter):
                header |= 1 << blocks
                put(prev)
                item_done()
        counter, prev = 1, v
    if counter >= 3:           # the last run: written, not counted
        put(bytes([counter]) + prev)
    else:
        for _ in range(counter):
            header |= 1 << blocks
            put(prev)
            item_done()
    return bytes(out[:pos])


def test_brle_trans4_encoder_matches_reference_writer():
    rng = np.random.default_rng(44)
    L = cc.lib()
    for trial in range(300):
        k = int(rng.integers(1, 5))
        words = np.repeat(rng.integers(0, k, 64), rng.integers(1, 12, 64))[:64]
        words = np.resize(words, 64).astype(np.uint32) * 0x01010101
        col = words.view(np.uint8)
        e = cc.brle_trans4_encode(_sym_column_chunk(col), 8192)
        r = int(np.nonzero(e.meta["col_map"][:32] == 0)[0][0])
        lanes, off = oracle.export_lanes(cc.Encoded("lzss", e.data, e.n_out, e.n_chunks, e.chunk_size, e.meta, {}))
        assert bytes(lanes[off[r]:off[r + 1]]) == _ref_compress_func_4B(col), trial


def _ref_compress_func_1B(col: np.ndarray) -> bytes:
    """brle_trans::compress_func of include/brle/brle_trans.h:437-562 for one
    column, restated loop for loop over an output zeroed beforehand: maximal
    runs, a run of 3 or more as (count, byte), shorter ones as literal bytes,
    a flag byte per 8 items, and the column's last run written without being
    counted (:529-536)."""
    out = bytearray(col.size * 2 + 16)
    pos = 1                    # byte_offset: header byte 0 reserved
    hdr, header, blocks = 0, 0, 0
    counter, prev = 0, None

    def item_done():
        nonlocal blocks, header, hdr, pos
        blocks += 1
        if blocks == 8:
            out[hdr] = header
            header = 0
            hdr = pos
            pos += 1
            blocks = 0
        if blocks != 0:
            out[hdr] = header

    def put(bs):
        nonlocal pos
        out[pos:pos + len(bs)] = bs
        pos += len(bs)

    for v in col.tolist():
        if counter == 0:
            prev = v
        if prev == v:
            counter += 1
            continue
        if counter >= 3:
            put(bytes([counter, prev]))
            item_done()
        else:
            for _ in range(counter):
                header |= 1 << blocks
                put(bytes([prev]))
                item_done()
        counter, prev = 1, v
    if counter >= 3:           # the last run: written, not counted
        put(bytes([counter, prev]))
    else:
        for _ in range(counter):
            header |= 1 << blocks
            put(bytes([prev]))
            item_done()
    return bytes(out[:pos])


def _byte_column_chunk(col: np.ndarray) -> np.ndarray:
    """A 4 KiB chunk whose column 0 holds `col` (128 bytes); the other
    columns are zero."""
    raw = np.zeros(4096, np.uint8)
    for k in range(32):
        raw[128 * k:128 * k + 4] = col[4 * k:4 * k + 4]
    return raw


def _column0_stream(e):
    r = int(np.nonzero(e.meta["col_map"][:32] == 0)[0][0])
    lanes, off = oracle.export_lanes(cc.Encoded("lzss", e.data, e.n_out, e.n_chunks, e.chunk_size, e.meta, {}))
    return bytes(lanes[off[r]:off[r + 1]]), int(e.meta["col_len"][r])


def test_brle_trans_last_run_in_slot_8():
    # 7 literal items, then a final run as the 8th item: written uncounted, so
    # no flag byte is reserved after it (col_len 1 + 7 + 2)
    col = np.array([1, 2, 3, 4, 5, 6, 7] + [9] * 121, np.uint8)
    e = cc.brle_trans_encode(_byte_column_chunk(col), 4096)
    stream, n = _column0_stream(e)
    assert n == 10 and stream == _ref_compress_func_1B(col)
    rc, out = oracle.decode(e)
    assert rc == 0 and np.array_equal(out, _byte_column_chunk(col))
    # 8 literal items end a group: the reserved flag byte follows them
    col = np.array([1, 2, 3, 4, 5, 6, 7, 8] + [9] * 120, np.uint8)
    e = cc.brle_trans_encode(_byte_column_chunk(col), 4096)
    stream, n = _column0_stream(e)
    assert n == 1 + 8 + 1 + 2 and stream == _ref_compress_func_1B(col)


def test_brle_trans_encoder_matches_reference_writer():
    rng = np.random.default_rng(45)
    for trial in range(400):
        k = int(rng.integers(1, 5))
        col = np.repeat(rng.integers(0, k, 128), rng.integers(1, 12, 128))[:128]
        col = np.resize(col, 128).astype(np.uint8)
        e = cc.brle_trans_encode(_byte_column_chunk(col), 4096)
        stream, n = _column0_stream(e)
        assert stream == _ref_compress_func_1B(col), trial
        assert n == len(stream)


def test_new_containers_reject_corruption():
    raw = cc.gen_markov_copy(5, 20000, 4096)
    e = cc.lzss_contig_encode(raw, 8192)
    cont = e.params["container"]
    cont[28 + 8 * e.n_chunks] ^= 1  # chunk 0's first token becomes a match with no history
    rc, _ = oracle.decode(e)
    assert rc != 0
    r2 = cc.gen_brle_bytes(6, 8192)
    e2 = cc.brle_trans_encode(r2, 4096)
    e2.meta["col_len"][0] -= 1  # truncated rank-0 stream
    rc, _ = oracle.decode(e2)
    assert rc != 0
