"""GPU parity: every sm_100a decoder, called through the C ABI, against the
CPU oracle on the same seeded inputs -- bit-exact, status OK -- plus
truncated/corrupted streams that must yield an error status (never a fault
or a hang: every device read and write is bounds checked)."""
import numpy as np
import pytest

import compression_b200.codecs as cc
import oracle

pytestmark = pytest.mark.gpu


def _gpu(enc, dev):
    import torch
    job = cc.DeviceJob(enc, dev)
    job.launch()
    torch.cuda.synchronize()
    return job.status(), job.output()


def _parity(enc, raw_bytes, dev):
    rc, ref = oracle.decode(enc)
    assert rc == 0 and np.array_equal(ref, raw_bytes)
    st, out = _gpu(enc, dev)
    assert (st == 0).all(), np.unique(st)
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("n", [1, 130, 256 * 1024, 256 * 1024 + 7, 5 * 256 * 1024 + 999])
def test_brle(cuda, n):
    raw = cc.gen_brle_bytes(n, n)
    _parity(cc.brle_encode(raw), raw, cuda)


def test_brle_patterns(cuda):
    rng = np.random.default_rng(0)
    for raw in [np.zeros(300000, np.uint8), np.arange(300000, dtype=np.uint8),
                rng.integers(0, 3, 700000).astype(np.uint8),
                np.repeat(rng.integers(0, 256, 3000), 200).astype(np.uint8)]:
        _parity(cc.brle_encode(raw, 65536), raw, cuda)


@pytest.mark.parametrize("eb,ccl", [(4, 128), (4, 16), (8, 64), (4, 256)])
def test_rlev1(cuda, eb, ccl):
    v = cc.gen_rlev1_ints(eb + ccl, 400000)
    raw = v.astype(np.int64) if eb == 8 else v
    enc = cc.rlev1_encode(raw, 32 * ccl * 8, ccl, eb)
    _parity(enc, raw.view(np.uint8), cuda)


def test_rlev1_config_chunk(cuda):
    v = cc.gen_rlev1_ints(11, 3 * 32768 + 100)
    _parity(cc.rlev1_encode(v, 128 * 1024, 128, 4), v.view(np.uint8), cuda)


@pytest.mark.parametrize("ru", [1, 4, 32, 64])
def test_rlev2(cuda, ru):
    v = cc.gen_rlev2_ints(ru, 200000)
    _parity(cc.rlev2_encode(v, 256 * ru * 4, ru), v.view(np.uint8), cuda)


def test_rlev2_wide_lanes_use_four_streams_per_block(cuda):
    """Lane streams too long for 8 per block in shared memory (1 MiB chunks of
    wide random values, about 30 KB per lane stream): the default launch
    falls back to 4 streams per block and still decodes as the oracle."""
    rng = np.random.default_rng(12)
    v = rng.integers(-2**59, 2**59, 3 * (1 << 17)).astype(np.int64)  # 3 chunks of 1 MiB
    enc = cc.rlev2_encode(v, 1 << 20, 32)
    assert 8 * (int(enc.meta["col_len"].max()) + 48) > 200 * 1024  # 8 streams would not fit
    _parity(enc, v.view(np.uint8), cuda)


def test_rlev2_negative_and_wide(cuda):
    rng = np.random.default_rng(1)
    v = np.concatenate([rng.integers(-2**62, 2**62, 3000), -np.arange(3000), np.full(500, -7),
                        rng.integers(0, 2**12, 3000) + (rng.random(3000) < 0.03) * 2**50]).astype(np.int64)
    _parity(cc.rlev2_encode(v, 256 * 8 * 2, 8), v.view(np.uint8), cuda)


@pytest.mark.parametrize("chunk", [128, 4096, 65536])
def test_lzss(cuda, chunk):
    raw = cc.gen_markov_copy(chunk, 5 * chunk, 4096)
    _parity(cc.lzss_encode(raw, chunk), raw, cuda)


def test_lzss_degenerate(cuda):
    for raw in [np.zeros(8192, np.uint8), np.tile(np.arange(7, dtype=np.uint8), 2000)[:8192]]:
        _parity(cc.lzss_encode(raw, 4096), raw, cuda)


@pytest.mark.parametrize("zh", [0, 1])
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_inflate(cuda, zh, mode):
    raw = cc.gen_markov_copy(9 + mode, 600000, 32768)
    oo = np.array([0, 1, 4097, 100000, 100000, 250000, 600000], dtype=np.uint64)
    _parity(cc.deflate_encode(raw, oo, 6, np.full(6, mode, np.uint8), zh), raw, cuda)


def test_inflate_many_uneven(cuda):
    raw = cc.gen_markov_copy(21, 8 << 20, 32768)
    sizes = cc.loguniform_sizes(22, 200, 4096, 1 << 20, raw.size)
    oo = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
    mode = (np.random.default_rng(3).random(200) < 0.05).astype(np.uint8)
    _parity(cc.deflate_encode(raw, oo, 6, mode), raw, cuda)


def test_host_api_matches(cuda):
    raw = cc.gen_brle_bytes(5, 700000)
    assert np.array_equal(cc.decode_host(cc.brle_encode(raw)), raw)
    v = cc.gen_rlev1_ints(6, 100000)
    assert np.array_equal(cc.decode_host(cc.rlev1_encode(v)), v.view(np.uint8))
    v2 = cc.gen_rlev2_ints(7, 100000)
    assert np.array_equal(cc.decode_host(cc.rlev2_encode(v2)), v2.view(np.uint8))
    raw3 = cc.gen_markov_copy(8, 4 * 65536, 4096)
    assert np.array_equal(cc.decode_host(cc.lzss_encode(raw3)), raw3)
    raw4 = cc.gen_markov_copy(9, 5 * 131072 + 77, 32768)
    oo = np.array([0, 131072, 262144, 393216, 524288, 655360, raw4.size], dtype=np.uint64)
    assert np.array_equal(cc.decode_host(cc.deflate_encode(raw4, oo)), raw4)


# ---------------------------------------------------------------------------
# malformed inputs: error status, no fault, no hang
# ---------------------------------------------------------------------------

def _expect_error(enc, dev):
    st, _ = _gpu(enc, dev)
    assert (st != 0).any()


def test_corrupt_brle(cuda):
    raw = cc.gen_brle_bytes(3, 600000)
    enc = cc.brle_encode(raw)
    enc.data[5] = 255          # literal header: extra output bytes
    _expect_error(enc, cuda)
    enc = cc.brle_encode(raw)
    enc.meta["ptr"][1] -= 1    # truncated chunk
    _expect_error(enc, cuda)


def test_corrupt_interleaved(cuda):
    v = cc.gen_rlev1_ints(4, 70000)
    enc = cc.rlev1_encode(v, 32 * 128 * 4, 128, 4)
    enc.meta["col_len"][3] = 2  # truncated lane
    _expect_error(enc, cuda)
    v2 = cc.gen_rlev2_ints(5, 40000)
    e2 = cc.rlev2_encode(v2, 256 * 32, 32)
    e2.meta["col_len"][0] += 1000000  # beyond the block
    _expect_error(e2, cuda)
    raw = cc.gen_markov_copy(6, 4 * 4096, 4096)
    e3 = cc.lzss_encode(raw, 4096)
    e3.meta["col_map"][1] = e3.meta["col_map"][0]  # not a permutation
    _expect_error(e3, cuda)
    e4 = cc.lzss_encode(raw, 4096)
    e4.data[:] = 0                                   # matches with offset 0
    _expect_error(e4, cuda)


def test_corrupt_inflate(cuda):
    raw = cc.gen_markov_copy(7, 300000, 32768)
    oo = np.array([0, 150000, 300000], dtype=np.uint64)
    enc = cc.deflate_encode(raw, oo)
    enc.meta["comp_len"][0] = 40   # truncated stream
    enc.data[int(enc.meta["comp_off"][1]) + 5] ^= 0xFF  # flipped bits
    _expect_error(enc, cuda)
    rng = np.random.default_rng(0)
    junk = cc.deflate_encode(raw, oo)
    junk.data[:] = rng.integers(0, 256, junk.data.size).astype(np.uint8)
    _expect_error(junk, cuda)


# ---------------------------------------------------------------------------
# containers built from the reference's own encoder output (tests/golden)
# ---------------------------------------------------------------------------

def test_reference_streams_on_gpu(cuda):
    from test_golden import _cases, interleave_streams
    # brle: the reference's container as is
    for raw, enc, _ in _cases("brle")[0]:
        n_ptr = int(enc[:4].view(np.uint32)[0])
        ptr = enc[4:4 + 8 * n_ptr].copy().view(np.uint64)
        e = cc.Encoded("brle", enc[4 + 8 * n_ptr + 8:].copy(), raw.size, n_ptr - 1, 256 * 1024, {"ptr": ptr})
        st, out = _gpu(e, cuda)
        assert (st == 0).all() and np.array_equal(out, raw)
    # LZSS: a 64 KiB chunk whose 32 columns are reference column streams
    cases = [c for c in _cases("lzss")[0] if c[0].size == 2048]
    cols = [cases[q % len(cases)] for q in range(32)]
    lens = np.array([c[1].size for c in cols])
    order = sorted(range(32), key=lambda q: (-lens[q], -q))  # rank: length desc, ties column desc
    blk, cl = interleave_streams([cols[q][1] for q in order])
    raw = np.zeros(65536, np.uint8)
    for q in range(32):
        raw.reshape(512, 32, 4)[:, q, :] = cols[q][0].reshape(512, 4)
    e = cc.Encoded("lzss", blk, raw.size, 1, 65536,
                   {"blk_off": np.array([0, blk.size], np.uint64), "col_len": cl,
                    "col_map": np.array(order, np.uint8)})
    st, out = _gpu(e, cuda)
    assert (st == 0).all() and np.array_equal(out, raw)
    # RLE v2: a 256 KiB chunk (READ_UNIT 32) whose lanes are reference streams
    cases = [c for c in _cases("rlev2")[0] if c[0].size == 1024]
    lanes = [cases[t % len(cases)] for t in range(32)]
    blk, cl = interleave_streams([l[1] for l in lanes])
    vals = np.zeros(32768, np.int64)
    for t in range(32):
        v = lanes[t][0]
        for k in range(32):
            vals[t * 32 + k * 1024: t * 32 + k * 1024 + 32] = v[k * 32:(k + 1) * 32]
    e = cc.Encoded("rlev2", blk, vals.nbytes, 1, 262144,
                   {"blk_off": np.array([0, blk.size], np.uint64), "col_len": cl}, {"read_unit": 32})
    st, out = _gpu(e, cuda)
    assert (st == 0).all() and np.array_equal(out, vals.view(np.uint8))


def test_reference_writer_containers_on_gpu(cuda):
    """Containers written by the reference's own GPU-only writers (RLE v1,
    byte-RLE flag with 1- and 4-byte symbols; tests/golden, produced by the
    reference kernels run on host threads) decode bit-exact on the device and
    agree with the reference's own reader."""
    from test_golden import _interleaved_cases
    for c in _interleaved_cases("rlev1"):
        eb, chunk, ccl = (int(x) for x in c["params"])
        e = cc.Encoded("rlev1", c["data"], c["raw"].size, c["blk_off"].size - 1, chunk,
                       {"blk_off": c["blk_off"], "col_len": c["col_len"]}, {"comp_col_len": ccl, "elem_bytes": eb})
        st, out = _gpu(e, cuda)
        assert (st == 0).all() and np.array_equal(out, c["raw"]) and np.array_equal(out, c["dec"])
    for name, chunk in (("brle_trans", 4096), ("brle_trans4", 8192)):
        for c in _interleaved_cases(name):
            e = cc.Encoded(name, c["data"], c["raw"].size, c["blk_off"].size - 1, chunk,
                           {"blk_off": c["blk_off"], "col_len": c["col_len"], "col_map": c["col_map"]})
            st, out = _gpu(e, cuda)
            assert (st == 0).all() and np.array_equal(out, c["raw"]) and np.array_equal(out, c["dec"]), name


# ---------------------------------------------------------------------------
# LZSS contiguous container and byte-RLE flag-byte container
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("n,chunk", [(1, 1024), (5000, 4096), (3 * 65536, 65536), (1 << 20, 128 * 1024),
                                     (700001, 128 * 1024)])
def test_lzss_contig(cuda, n, chunk):
    raw = cc.gen_markov_copy(n, n, 4096)
    _parity(cc.lzss_contig_encode(raw, chunk), raw, cuda)


def test_lzss_contig_patterns(cuda):
    rng = np.random.default_rng(2)
    for raw in [np.zeros(200000, np.uint8), rng.integers(0, 256, 200000).astype(np.uint8),
                np.tile(np.arange(11, dtype=np.uint8), 20000)]:
        _parity(cc.lzss_contig_encode(raw, 65536), raw, cuda)


@pytest.mark.parametrize("n,chunk", [(128, 128), (4096 * 300, 4096), (4096 * 7 + 1000, 4096), (8192 * 33, 8192),
                                     (1024 * 77, 1024)])
def test_brle_trans(cuda, n, chunk):
    raw = cc.gen_brle_bytes(n + chunk, n)
    _parity(cc.brle_trans_encode(raw, chunk), raw, cuda)


def test_brle_trans_patterns(cuda):
    rng = np.random.default_rng(4)
    for raw in [np.zeros(64 * 4096, np.uint8), rng.integers(0, 256, 64 * 4096).astype(np.uint8),
                np.repeat(rng.integers(0, 4, 32768), 8).astype(np.uint8)]:
        _parity(cc.brle_trans_encode(raw, 4096), raw, cuda)


def _word_runs(seed, n):
    rng = np.random.default_rng(seed)
    words = np.repeat(rng.integers(0, 6, n // 40 + 1), rng.integers(1, 20, n // 40 + 1)).astype(np.uint32)
    return np.resize(words, (n + 3) // 4).view(np.uint8)[:n].copy()


@pytest.mark.parametrize("n,chunk", [(8192 * 300, 8192), (8192 * 5 + 100, 8192), (4096 * 33, 4096), (128 * 50, 128)])
def test_brle_trans4(cuda, n, chunk):
    _parity(cc.brle_trans4_encode(_word_runs(n, n), chunk), _word_runs(n, n), cuda)
    rng = np.random.default_rng(n)
    for raw in [np.zeros(n, np.uint8), rng.integers(0, 256, n).astype(np.uint8)]:
        _parity(cc.brle_trans4_encode(raw, chunk), raw, cuda)


def test_brle_trans4_host_api_and_corruption(cuda):
    raw = _word_runs(3, 8192 * 40 + 17)
    out = cc.decode_host(cc.brle_trans4_encode(raw, 8192))
    # like the reference's decompress_gpu, the host call returns whole chunks
    # (the last one zero-padded)
    assert out.size == 8192 * 41 and np.array_equal(out[:raw.size], raw) and not out[raw.size:].any()
    e = cc.brle_trans4_encode(raw, 8192)
    e.meta["col_len"][0] -= 1  # truncated rank-0 stream: an item cut short
    _expect_error(e, cuda)
    e = cc.brle_trans4_encode(raw, 8192)
    e.meta["col_map"][1] = e.meta["col_map"][0]  # not a permutation
    _expect_error(e, cuda)


def test_new_containers_host_api(cuda):
    raw = cc.gen_markov_copy(8, 5 * 65536 + 333, 4096)
    assert np.array_equal(cc.decode_host(cc.lzss_contig_encode(raw, 65536)), raw)
    raw2 = cc.gen_brle_bytes(9, 4096 * 40)
    assert np.array_equal(cc.decode_host(cc.brle_trans_encode(raw2, 4096)), raw2)


def test_new_containers_corrupt(cuda):
    raw = cc.gen_markov_copy(5, 200000, 4096)
    e = cc.lzss_contig_encode(raw, 8192)
    e.data[0] ^= 1  # chunk 0's first token becomes a match with no history
    _expect_error(e, cuda)
    e = cc.lzss_contig_encode(raw, 8192)
    e.meta["ends"][3] -= 1  # chunk 3 truncated, chunk 4 starts one byte early
    _expect_error(e, cuda)
    r2 = cc.gen_brle_bytes(6, 4096 * 8)
    e2 = cc.brle_trans_encode(r2, 4096)
    e2.meta["col_len"][0] -= 1  # truncated rank-0 stream
    _expect_error(e2, cuda)
    e3 = cc.brle_trans_encode(r2, 4096)
    e3.meta["col_map"][1] = e3.meta["col_map"][0]  # not a permutation
    _expect_error(e3, cuda)
    e4 = cc.brle_trans_encode(r2, 4096)
    e4.meta["col_len"][32] = 10_000  # longer than any valid column stream
    _expect_error(e4, cuda)


def _lzss_token_column(rng, col_bytes):
    """One LZSS column stream with every token shape the grammar allows:
    literals, matches of length 3..34 at offsets 1..o, including offsets below
    the length (the source overlaps the output, copied byte by byte)."""
    toks, o = [], 0
    while o < col_bytes:
        if o == 0 or rng.random() < 0.35:
            toks.append(("l", int(rng.integers(0, 256))))
            o += 1
            continue
        ln = int(min(rng.integers(3, 35), col_bytes - o))
        if ln < 3:
            toks.append(("l", int(rng.integers(0, 256))))
            o += 1
            continue
        r = rng.random()
        off = int(rng.integers(1, 4)) if r < 0.25 else int(rng.integers(4, 9)) if r < 0.45 else \
            int(rng.integers(1, o + 1))
        off = min(off, o)
        toks.append(("m", off, ln))
        o += ln
    out = bytearray()
    for g in range(0, len(toks), 8):
        grp = toks[g:g + 8]
        out.append(sum(1 << i for i, t in enumerate(grp) if t[0] == "l"))
        for t in grp:
            if t[0] == "l":
                out.append(t[1])
            else:
                v = (t[1] << 5) | (t[2] - 3)
                out += bytes([v & 0xFF, v >> 8])
    return np.frombuffer(bytes(out), np.uint8)


@pytest.mark.parametrize("knob", [0, 4, 512, 256, 1])
@pytest.mark.parametrize("chunk", [4096, 65536])
def test_lzss_token_shapes(cuda, knob, chunk):
    from test_golden import interleave_streams
    import compression_b200.autotune as at
    rng = np.random.default_rng(chunk + knob)
    blocks, cls, maps = [], [], []
    for c in range(3):
        cols = [_lzss_token_column(rng, chunk // 32) for _ in range(32)]
        order = sorted(range(32), key=lambda q: -cols[q].size)
        blk, cl = interleave_streams([cols[q] for q in order])
        blocks.append(blk)
        cls.append(cl)
        maps.append(np.array(order, np.uint8))
    bo = np.concatenate([[0], np.cumsum([b.size for b in blocks])]).astype(np.uint64)
    e = cc.Encoded("lzss", np.concatenate(blocks), 3 * chunk, 3, chunk,
                   {"blk_off": bo, "col_len": np.concatenate(cls), "col_map": np.concatenate(maps)})
    rc, ref = oracle.decode(e)
    assert rc == 0
    prev = at.set_knob(at.TUNE_LZSS_WARPS_PER_BLOCK, knob)
    try:
        st, out = _gpu(e, cuda)
    finally:
        at.set_knob(at.TUNE_LZSS_WARPS_PER_BLOCK, prev)
    assert (st == 0).all(), np.unique(st)
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14])
def test_inflate_variants(cuda, variant):
    """Every inflate kernel shape on streams of mixed size with dynamic,
    fixed-Huffman and stored blocks, against zlib."""
    import compression_b200.autotune as at
    raw = cc.gen_markov_copy(11, 3 << 20, 32768)
    sizes = cc.loguniform_sizes(12, 40, 1024, 256 * 1024, raw.size)
    oo = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
    mode = (np.arange(40) % 7 == 3).astype(np.uint8) + 2 * (np.arange(40) % 11 == 5).astype(np.uint8)
    enc = cc.deflate_encode(raw[: int(oo[-1])], oo, 6, mode, 1)
    prev = at.set_knob(at.TUNE_INFLATE_VARIANT, variant)
    try:
        _parity(enc, raw[: int(oo[-1])], cuda)
    finally:
        at.set_knob(at.TUNE_INFLATE_VARIANT, prev)


def test_host_calls_in_many_pieces(cuda):
    """Host calls large enough to run as many overlapped pieces (each at
    least 4 MiB of output): byte-exact, for every codec, with pinned and
    pageable input; Deflate streams of uneven size (longest first inside each
    piece) and a last chunk that is short."""
    raw = cc.gen_brle_bytes(21, 40 * (1 << 20) + 12345)
    assert np.array_equal(cc.decode_host(cc.brle_encode(raw)), raw)
    v1 = cc.gen_rlev1_ints(22, 9 * (1 << 20) // 4)
    e1 = cc.rlev1_encode(v1, 128 * 1024, 128, 4)
    assert np.array_equal(cc.decode_host(e1), v1.view(np.uint8))
    cc.decode_host_pinned(e1)  # the pinned path runs without error
    v2 = cc.gen_rlev2_ints(23, 40 * (1 << 20) // 8)
    assert np.array_equal(cc.decode_host(cc.rlev2_encode(v2, 256 * 1024, 32)), v2.view(np.uint8))
    lz = cc.gen_markov_copy(24, 40 * (1 << 20), 4096)
    assert np.array_equal(cc.decode_host(cc.lzss_encode(lz, 64 * 1024)), lz)
    bt = cc.gen_brle_bytes(25, 20 * (1 << 20))
    assert np.array_equal(cc.decode_host(cc.brle_trans_encode(bt, 4096)), bt)
    d = cc.gen_markov_copy(26, 48 * (1 << 20), 32768)
    sizes = cc.loguniform_sizes(27, 300, 4096, 1 << 20, d.size)
    oo = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
    ed = cc.deflate_encode(d[: int(oo[-1])], oo)
    assert np.array_equal(cc.decode_host(ed), d[: int(oo[-1])])
    n9 = 9 * (1 << 20) + 5  # uniform 1 MiB chunks (the reference's container) and a 5-byte last one
    oo9 = np.array(list(range(0, 9 * (1 << 20) + 1, 1 << 20)) + [n9], dtype=np.uint64)
    assert np.array_equal(cc.decode_host(cc.deflate_encode(d[:n9], oo9)), d[:n9])


@pytest.mark.parametrize("knob", [4, 8])
def test_rlev2_decoder_shapes(cuda, knob):
    """Both RLE v2 kernel shapes (4 / 8 lane streams per block) on all four run kinds, signed and 64-bit-wide values, wide
    patches, a short last chunk, READ_UNIT 8 / 32 / 64 and the reference
    encoder's fixed-delta quirk, against the oracle; corrupt streams fail."""
    import compression_b200.autotune as at
    rng = np.random.default_rng(knob)
    v = np.concatenate([rng.integers(-2**62, 2**62, 3000), -np.arange(3000), np.full(500, -7),
                        rng.integers(0, 2**12, 3000) + (rng.random(3000) < 0.03) * 2**50,
                        cc.gen_rlev2_ints(knob, 40000)]).astype(np.int64)
    prev = at.set_knob(at.TUNE_RLEV2_LANES_PER_BLOCK, knob)
    try:
        for ru in (8, 32, 64):
            enc = cc.rlev2_encode(v, 256 * ru * 4, ru)
            rc, ref = oracle.decode(enc)
            assert rc == 0
            st, out = _gpu(enc, cuda)
            assert (st == 0).all(), np.unique(st)
            assert np.array_equal(out, ref)
        quirk = cc.gen_rlev2_ints(0xE0 * 100003 + 9149, 5120 * 8)
        enc = cc.rlev2_encode(quirk, 256 * 32, 32)
        rc, ref = oracle.decode(enc)
        st, out = _gpu(enc, cuda)
        assert rc == 0 and (st == 0).all() and np.array_equal(out, ref)
        bad = cc.rlev2_encode(cc.gen_rlev2_ints(5, 40000), 256 * 32, 32)
        bad.meta["col_len"][0] += 1000000  # beyond the block
        st, _ = _gpu(bad, cuda)
        assert (st != 0).any()
        bad2 = cc.rlev2_encode(cc.gen_rlev2_ints(6, 40000), 256 * 32, 32)
        bad2.data[: bad2.data.size // 2] = 0xFF  # garbage headers
        st, _ = _gpu(bad2, cuda)
        assert (st != 0).any()
    finally:
        at.set_knob(at.TUNE_RLEV2_LANES_PER_BLOCK, prev)


def _lzss_pack(toks):
    """Token list (("l", byte) or ("m", offset, length)) -> LZSS column stream."""
    out = bytearray()
    for g in range(0, len(toks), 8):
        grp = toks[g:g + 8]
        out.append(sum(1 << i for i, t in enumerate(grp) if t[0] == "l"))
        for t in grp:
            if t[0] == "l":
                out.append(t[1])
            else:
                v = (t[1] << 5) | (t[2] - 3)
                out += bytes([v & 0xFF, v >> 8])
    return np.frombuffer(bytes(out), np.uint8)


def _lzss_tokens_ending_in_match(rng, col_bytes):
    toks, o = [], 0
    while o < col_bytes - 8:
        if o < 4 or col_bytes - 8 - o < 3 or rng.random() < 0.6:
            toks.append(("l", int(rng.integers(0, 256))))
            o += 1
        else:
            ln = int(rng.integers(3, min(35, col_bytes - 8 - o + 1)))
            toks.append(("m", int(rng.integers(1, min(o, 2047) + 1)), ln))
            o += ln
    while o < col_bytes - 5:
        toks.append(("l", int(rng.integers(0, 256))))
        o += 1
    toks.append(("m", int(rng.integers(1, o + 1)), col_bytes - o))  # the last token: a match up to the end
    return toks


def test_lzss_corrupt_statuses_agree(cuda):
    """One planted defect per chunk (truncated column, offset past the column
    start, offset 0, a last match running past the column end): every LZSS
    kernel choice reports the oracle's status for every chunk, and the clean
    chunk decodes as the oracle does."""
    from test_golden import interleave_streams
    import compression_b200.autotune as at
    rng = np.random.default_rng(77)
    chunk = 65536
    cb = chunk // 32
    blocks, cls, maps = [], [], []
    for c in range(5):
        cols = []
        for q in range(32):
            toks = _lzss_tokens_ending_in_match(rng, cb)
            if c == 2 and q == 7:    # first match reaches before the column start
                i = next(k for k, t in enumerate(toks) if t[0] == "m")
                o = sum(1 if t[0] == "l" else t[2] for t in toks[:i])
                toks[i] = ("m", o + 1, toks[i][2])
            if c == 3 and q == 9:    # the last match runs 3 bytes past the column end
                toks[-1] = ("m", toks[-1][1], toks[-1][2] + 3)
            if c == 4 and q == 20:   # a match with offset 0
                i = next(k for k, t in enumerate(toks) if t[0] == "m")
                toks[i] = ("m", 0, toks[i][2])
            s = _lzss_pack(toks)
            if c == 1 and q == 5:    # truncated: the stream ends inside its last match
                s = s[:-1]
            cols.append(s)
        order = sorted(range(32), key=lambda q: -cols[q].size)
        blk, cl = interleave_streams([cols[q] for q in order])
        blocks.append(blk)
        cls.append(cl)
        maps.append(np.array(order, np.uint8))
    # the oracle's status of every chunk alone
    want, ref = [], None
    for c in range(5):
        one = cc.Encoded("lzss", blocks[c].copy(), chunk, 1, chunk,
                         {"blk_off": np.array([0, blocks[c].size], np.uint64), "col_len": cls[c], "col_map": maps[c]})
        rc, out = oracle.decode(one)
        want.append(rc)
        if c == 0:
            ref = out
    assert want == [0, 2, 2, 3, 2]  # GD_OK, GD_ERR_CORRUPT x2, GD_ERR_OVERRUN, GD_ERR_CORRUPT
    bo = np.concatenate([[0], np.cumsum([b.size for b in blocks])]).astype(np.uint64)
    e = cc.Encoded("lzss", np.concatenate(blocks), 5 * chunk, 5, chunk,
                   {"blk_off": bo, "col_len": np.concatenate(cls), "col_map": np.concatenate(maps)})
    for knob in (0, 4, 512, 256, 1):
        prev = at.set_knob(at.TUNE_LZSS_WARPS_PER_BLOCK, knob)
        try:
            st, out = _gpu(e, cuda)
        finally:
            at.set_knob(at.TUNE_LZSS_WARPS_PER_BLOCK, prev)
        assert list(st) == want, (knob, list(st))
        assert np.array_equal(out[:chunk], ref), knob
