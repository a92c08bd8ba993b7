"""GPU parity of the byte-RLE, byte-RLE flag, LZSS, RLE v1 and RLE v2 device
encoders: the container written on the device is byte-identical to the host
encoder's, whose streams are pinned against the reference's own encoders in
test_golden.py, and decodes back to the column through the device decoder
and the oracle."""
import numpy as np
import pytest

import compression_b200.codecs as cc
import oracle

pytestmark = pytest.mark.gpu


def _same(a: cc.Encoded, b: cc.Encoded):
    assert a.n_chunks == b.n_chunks
    assert np.array_equal(a.meta["blk_off"], b.meta["blk_off"])
    assert np.array_equal(a.meta["col_len"], b.meta["col_len"])
    assert np.array_equal(a.data, b.data)
    if "col_map" in b.meta:
        assert np.array_equal(a.meta["col_map"], b.meta["col_map"])


def _roundtrip(enc: cc.Encoded, raw_bytes: np.ndarray, dev, exact: bool = True):
    """The device decoder returns what the oracle decodes; with exact, that
    is the column itself.  Some RLE v2 inputs do not round-trip through the
    reference's own encoder: constant runs after short repeats written as
    fixed-delta runs with a non-zero delta (parity is then with the reference
    decoder), and 128-value runs of a negative constant written as a corrupt
    DIRECT header (both decoders report an error)."""
    import torch
    rc, ref = oracle.decode(enc)
    job = cc.DeviceJob(enc, dev)
    job.launch()
    torch.cuda.synchronize()
    if rc != 0:  # a stream the reference's encoder writes corrupt: both decoders say so
        assert not exact and (job.status() != 0).any()
        return
    if exact:
        assert np.array_equal(ref, raw_bytes)
    assert (job.status() == 0).all()
    assert np.array_equal(job.output(), ref)


def _rlev1_inputs(eb):
    rng = np.random.default_rng(eb)
    t = np.uint32 if eb == 4 else np.uint64
    yield cc.gen_rlev1_ints(eb, 300000).astype(t)
    yield rng.integers(0, 2**63 if eb == 8 else 2**32, 200000, dtype=np.uint64).astype(t)  # literals only
    yield np.full(150000, 7, t)                                                           # runs only
    yield (np.arange(180000) * 3 - 1000).astype(t)                                        # fixed deltas, wrap
    yield np.repeat(rng.integers(0, 300, 4000), rng.integers(1, 6, 4000)).astype(t)      # short runs
    v = rng.integers(0, 1 << 20, 100000).astype(t)
    v[::7] = v[1::7][: v[::7].size]                                                      # 2-value repeats
    yield v


@pytest.mark.parametrize("eb,ccl,chunk", [(4, 128, 128 * 1024), (4, 4, 4096), (4, 32, 32 * 1024),
                                          (8, 64, 64 * 1024), (8, 8, 8192), (4, 256, 32 * 1024)])
def test_rlev1_device_encoder(cuda, eb, ccl, chunk):
    for v in _rlev1_inputs(eb):
        raw = v.view(np.uint8)
        host = cc.rlev1_encode(raw, chunk, ccl, eb)
        dev = cc.encode_gpu("rlev1", raw, chunk, comp_col_len=ccl, elem_bytes=eb)
        _same(dev, host)
        _roundtrip(dev, raw, cuda)


def _rlev2_inputs():
    rng = np.random.default_rng(2)
    yield cc.gen_rlev2_ints(5, 300000)
    yield rng.integers(-2**63, 2**63 - 1, 100000, dtype=np.int64)          # 64-bit DIRECT
    yield np.full(70000, 5, np.int64)                                      # constant runs
    yield np.full(70000, -5, np.int64)  # negative: corrupt in the reference encoder (negconst fixture)
    yield np.cumsum(rng.integers(1, 1000, 90000)).astype(np.int64)         # DELTA
    yield (np.cumsum(rng.integers(-3, 4, 90000)) * 1000).astype(np.int64)  # signed deltas
    v = rng.integers(0, 1 << 12, 120000).astype(np.int64)
    v[rng.random(v.size) < 0.02] = rng.integers(0, 1 << 40, 1)[0]           # PATCHED_BASE
    yield v
    yield np.repeat(rng.integers(-1 << 40, 1 << 40, 20000), rng.integers(1, 14, 20000)).astype(np.int64)


@pytest.mark.parametrize("ru,chunk", [(32, 256 * 1024), (1, 8192), (4, 4 * 4096), (64, 64 * 1024)])
def test_rlev2_device_encoder(cuda, ru, chunk):
    for i, v in enumerate(_rlev2_inputs()):
        raw = v.view(np.uint8)
        host = cc.rlev2_encode(raw, chunk, ru)
        dev = cc.encode_gpu("rlev2", raw, chunk, read_unit=ru)
        _same(dev, host)
        _roundtrip(dev, raw, cuda, exact=i not in (3, 7))


def _brle_inputs():
    rng = np.random.default_rng(7)
    yield cc.gen_brle_bytes(1, 700000)
    yield np.zeros(300000, np.uint8)                                   # one long run
    yield rng.integers(0, 256, 200000).astype(np.uint8)                # incompressible: one region
    yield rng.integers(0, 2, 300000).astype(np.uint8)                  # short runs
    yield np.arange(100000, dtype=np.uint8)
    for L in (5, 129, 130, 131, 133, 134, 135, 260, 261, 264, 265):   # run lengths around 130 multiples
        pieces = []
        for _ in range(400):
            pieces.append(np.full(L if rng.random() < 0.5 else int(rng.integers(1, 7)), int(rng.integers(0, 4)),
                                  np.uint8))
            pieces.append(rng.integers(0, 256, int(rng.integers(0, 140))).astype(np.uint8))
        yield np.concatenate(pieces)
    pieces = []                                                         # runs right after 126..129 literals
    for _ in range(500):
        pieces.append((np.arange(int(rng.integers(120, 135))) * 3 % 251).astype(np.uint8))
        pieces.append(np.full(int(rng.integers(3, 300)), 255, np.uint8))
    yield np.concatenate(pieces)
    for n in (1, 2, 3, 100, 255, 257, 4097):
        yield cc.gen_brle_bytes(n, n)


@pytest.mark.parametrize("chunk", [256 * 1024, 65536, 4096, 1000])
def test_brle_device_encoder(cuda, chunk):
    for raw in _brle_inputs():
        host = cc.brle_encode(raw, chunk)
        dev = cc.encode_gpu("brle", raw, chunk)
        assert np.array_equal(dev.params["container"], host.params["container"])
        _roundtrip(dev, raw, cuda)


@pytest.mark.parametrize("chunk", [4096, 128, 1024, 8064])
def test_brle_trans_device_encoder(cuda, chunk):
    for raw in _brle_inputs():
        host = cc.brle_trans_encode(raw, chunk)
        dev = cc.encode_gpu("brle_trans", raw, chunk)
        _same(dev, host)
        _roundtrip(dev, raw, cuda)


def _lzss_inputs():
    rng = np.random.default_rng(11)
    yield cc.gen_markov_copy(3, 1 << 20, 4096)
    yield np.zeros(300000, np.uint8)                                    # 34-byte matches everywhere
    yield rng.integers(0, 256, 200000).astype(np.uint8)                 # literals only
    yield np.tile(np.arange(7, dtype=np.uint8), 40000)
    yield rng.integers(0, 4, 300000).astype(np.uint8)                   # long candidate lists, short matches
    yield (np.arange(300000) // 64 % 5).astype(np.uint8)
    yield cc.gen_markov_copy(4, 100003, 4096)                           # a short last chunk


@pytest.mark.parametrize("chunk", [64 * 1024, 128 * 1024, 4096, 128])
def test_lzss_device_encoder(cuda, chunk):
    for raw in _lzss_inputs():
        host = cc.lzss_encode(raw, chunk)
        dev = cc.encode_gpu("lzss", raw, chunk)
        _same(dev, host)
        _roundtrip(dev, raw, cuda)


def test_device_encoders_at_bench_sizes(cuda):
    """Full-size columns (256 MiB byte-RLE, 64 MiB int32 RLE v1, 256 MiB
    int64 RLE v2; 256 MiB of the LZSS column): the device container equals
    the host encoder's, and the device decoder returns what the oracle
    decodes."""
    raw = cc.gen_brle_bytes(0xB0, 256 << 20)
    dev = cc.encode_gpu("brle", raw, 256 * 1024)
    assert np.array_equal(dev.params["container"], cc.brle_encode(raw, 256 * 1024).params["container"])
    _roundtrip(dev, raw, cuda)
    raw = cc.gen_markov_copy(0xC0, 256 << 20, 4096)                     # LZSS: a quarter of the 1 GiB column
    dev = cc.encode_gpu("lzss", raw, 64 * 1024)
    _same(dev, cc.lzss_encode(raw, 64 * 1024))
    _roundtrip(dev, raw, cuda)
    v1 = cc.gen_rlev1_ints(0xA0, (64 << 20) // 4)
    v2 = cc.gen_rlev2_ints(0xB0, (256 << 20) // 8)
    for codec, v, kw, host in (
            ("rlev1", v1, dict(comp_col_len=128, elem_bytes=4), lambda r: cc.rlev1_encode(r, 128 * 1024, 128, 4)),
            ("rlev2", v2, dict(read_unit=32), lambda r: cc.rlev2_encode(r, 256 * 1024, 32))):
        raw = v.view(np.uint8)
        chunk = 128 * 1024 if codec == "rlev1" else 256 * 1024
        dev = cc.encode_gpu(codec, raw, chunk, **kw)
        _same(dev, host(raw))
        _roundtrip(dev, raw, cuda, exact=codec == "rlev1")


def test_device_encoder_argument_errors(cuda):
    import torch
    d = torch.zeros(1000, dtype=torch.uint8, device=cuda)
    with pytest.raises(cc.DecodeError):
        cc.encode_device("rlev1", d[:999], 4096, comp_col_len=128, elem_bytes=4)   # not whole values
    with pytest.raises(cc.DecodeError):
        cc.encode_device("rlev1", d, 4000, comp_col_len=128, elem_bytes=4)        # chunk not 32 slices
    with pytest.raises(cc.DecodeError):
        cc.encode_device("rlev2", d[:996], 8192, read_unit=1)                     # not whole int64 values
    with pytest.raises(cc.DecodeError):
        cc.encode_device("rlev2", d, 8192, read_unit=3)                           # chunk % (256 * ru)
    with pytest.raises(cc.DecodeError):
        cc.encode_device("brle", d, 1 << 31)                                      # chunk above 1 GiB
    with pytest.raises(cc.DecodeError):
        cc.encode_device("lzss", d, 1000)                                         # chunk not 128-byte rows
    with pytest.raises(cc.DecodeError):
        cc.encode_device("lzss", d, 256 * 1024)                                   # column above 4 KiB
    with pytest.raises(cc.DecodeError):
        cc.encode_device("brle_trans", d, 8192)                                   # column above 252 bytes


def test_host_compress_calls(cuda):
    """gd_brle_compress / gd_rlev1_compress / gd_rlev2_compress /
    gd_lzss_compress (the reference's compress_gpu calls, host buffers in
    and out): the same container and metadata as the host encoders, and the
    host decompress call returns the column."""
    raw = cc.gen_brle_bytes(5, 3_000_001)
    dev = cc.compress_host("brle", raw)
    assert np.array_equal(dev.params["container"], cc.brle_encode(raw).params["container"])
    assert np.array_equal(cc.decode_host(dev), raw)
    raw = cc.gen_markov_copy(6, 1_000_003, 4096)
    dev = cc.compress_host("lzss", raw)
    _same(dev, cc.lzss_encode(raw, 128 * 1024))
    assert dev.chunk_size == 128 * 1024
    assert np.array_equal(cc.decode_host(dev)[:raw.size], raw)
    for eb, ccl, chunk in ((4, 128, 128 * 1024), (8, 64, 64 * 1024)):
        v = cc.gen_rlev1_ints(eb, 700_001).astype(np.uint32 if eb == 4 else np.uint64)
        raw = v.view(np.uint8)
        dev = cc.compress_host("rlev1", raw, chunk, comp_col_len=ccl, elem_bytes=eb)
        _same(dev, cc.rlev1_encode(raw, chunk, ccl, eb))
        assert int(dev.params["container"][:8].view(np.uint64)[0]) == raw.size
        assert np.array_equal(cc.decode_host(dev), raw)
    for ru, chunk in ((32, 256 * 1024), (4, 4 * 4096)):
        raw = cc.gen_rlev2_ints(7, 500_001).view(np.uint8)
        dev = cc.compress_host("rlev2", raw, chunk, read_unit=ru)
        _same(dev, cc.rlev2_encode(raw, chunk, ru))
        assert np.array_equal(cc.decode_host(dev), raw)
    # twice in a row on the same thread: the staging pool is reused
    raw = cc.gen_brle_bytes(8, 100_000)
    a, b = cc.compress_host("brle", raw), cc.compress_host("brle", raw)
    assert np.array_equal(a.params["container"], b.params["container"])
