// lzss.cuh -- warp-level LZSS chunk decoder (shared by the plain kernel in
// lzss.cu and the batched decoder in batch.cu).
//
// Grammar (restated from lzss::decompress_func, include/lzss/lzss_gpu2.h:
// 112-325): per column stream, a flag byte then 8 tokens LSB-first; flag 1 =
// one literal byte, flag 0 = little-endian 16-bit v with length (v & 31) + 3
// and offset v >> 5 back into this column's own output.  Column q of a chunk
// owns output bytes 4q + 128k .. +3.  The streams are ranked by descending
// length (col_len sorted, col_map = rank -> column) and 4-byte interleaved.
//
// The reference runs one thread per column with a 2 KiB history array in
// local memory and byte-wise 4-byte-strided stores.  Here a warp decodes a
// chunk (lane = rank) with the shared interleave reader; each round every
// lane produces 64 bytes (16 output rows) of its column into shared memory,
// then the warp writes those 16 rows (2 KiB contiguous) with coalesced
// stores.  Match sources inside the current round come from shared memory,
// older ones from the already-written output (same SM, ordered by
// __syncwarp).  A match never overlaps its source (length <= offset,
// lzss_gpu2.h:79), but the byte loop is correct either way.
#pragma once
#include "interleave.cuh"

namespace gd {
namespace lzss {

constexpr uint32_t RB = 64;        // column bytes per lane per round (16 rows)
constexpr uint32_t SSTR = RB + 4;  // 17 words: row reads across columns are conflict-free
constexpr uint32_t WARP_SMEM = (uint32_t)sizeof(SegTable) + 32u * RING_STRIDE + 32u * SSTR;

// Decode one LZSS chunk with the calling warp.  `block` = the chunk's
// interleaved block (b_len bytes, 4-byte aligned), col_len/col_map = its 32
// rank entries, cout = its output (chunk_size bytes, 4-byte aligned),
// wsmem = WARP_SMEM bytes of shared memory owned by this warp.
// Returns a gd status; every lane returns the same value.
static __device__ __noinline__ uint32_t chunk_warp(const uint8_t* __restrict__ block, uint64_t b_len,
                                            const uint64_t* __restrict__ col_len,
                                            const uint8_t* __restrict__ col_map, uint64_t chunk_size,
                                            uint8_t* cout, uint8_t* wsmem) {
    const uint32_t lane = lane_id();
    SegTable* T_ = reinterpret_cast<SegTable*>(wsmem);
    uint8_t* ring = wsmem + sizeof(SegTable);
    uint8_t* stage = ring + 32 * RING_STRIDE;

    uint32_t err = ST_OK;
    const uint64_t len64 = col_len[lane];
    const uint32_t len = len64 > 0x3fffffffull ? 0u : (uint32_t)len64;
    if (len64 > 0x3fffffffull) err = ST_CORRUPT;
    const uint32_t q = col_map[lane];
    if (q >= 32) err = ST_CORRUPT;
    {  // col_map must be a permutation of the 32 columns
        uint32_t bits = 0;
#pragma unroll
        for (int o = 0; o < 32; ++o) bits |= 1u << (__shfl_sync(GD_FULL_MASK, q, o) & 31u);
        if (bits != 0xffffffffu) err = ST_CORRUPT;
    }
    const uint32_t nw = (len + 3) >> 2;
    uint32_t tot = warp_incl_scan(nw);
    tot = __shfl_sync(GD_FULL_MASK, tot, 31);
    if ((uint64_t)tot * 4 > b_len) err = ST_CORRUPT;
    if ((reinterpret_cast<uintptr_t>(block) & 3u) != 0) err = ST_CORRUPT;  // words are 4-byte loads
    if (chunk_size == 0 || chunk_size % 128 || chunk_size > (1ull << 31)) err = ST_INVALID;
    if (__any_sync(GD_FULL_MASK, err != ST_OK)) return __reduce_max_sync(GD_FULL_MASK, err);
    seg_build(T_, nw);
    LaneWords lw;
    lw_init(lw, T_, nw);
    LaneRing r{ring + lane * RING_STRIDE, 0, 0, len};

    const uint32_t col_bytes = (uint32_t)(chunk_size / 32);
    const uint32_t rounds = (col_bytes + RB - 1) / RB;
    uint8_t* my_stage = stage + q * SSTR;
    uint32_t o = 0;            // column bytes produced
    uint32_t flags = 0, ntok = 0;
    uint32_t mrem = 0, msrc = 0;  // pending match: bytes left, source position

    auto rd_byte = [&](uint32_t& b) -> bool {
        if (r.rd >= r.len) return false;
        b = ring_byte(r, r.rd);
        ++r.rd;
        return true;
    };

    for (uint32_t rnd = 0; rnd < rounds; ++rnd) {
        const uint32_t r0 = rnd * RB;
        const uint32_t rend = min(r0 + RB, col_bytes);
        for (;;) {
            const bool act = (o < rend) && (err == ST_OK);
            const bool need = act && (r.fl - r.rd < (uint32_t)RING_LOW) && (lw.k < lw.nw);
            if (__any_sync(GD_FULL_MASK, need)) ring_refill(r, lw, T_, block);
            if (!__any_sync(GD_FULL_MASK, act)) break;
            if (!act) continue;
            uint32_t b = 0;
            if (mrem == 0) {
                if (ntok == 0) {
                    if (!rd_byte(flags)) {
                        err = ST_CORRUPT;
                        continue;
                    }
                    ntok = 8;
                }
                const uint32_t lit = flags & 1u;
                flags >>= 1;
                --ntok;
                if (lit) {
                    if (!rd_byte(b)) {
                        err = ST_CORRUPT;
                        continue;
                    }
                    my_stage[o - r0] = (uint8_t)b;
                    ++o;
                    continue;
                }
                uint32_t lo8, hi8;
                if (!rd_byte(lo8) || !rd_byte(hi8)) {
                    err = ST_CORRUPT;
                    continue;
                }
                const uint32_t v = lo8 | (hi8 << 8);
                const uint32_t mlen = (v & 31u) + 3u, off = v >> 5;
                if (off == 0 || off > o) {
                    err = ST_CORRUPT;
                    continue;
                }
                if (o + mlen > col_bytes) {
                    err = ST_OVERRUN;
                    continue;
                }
                mrem = mlen;
                msrc = o - off;
            }
            // one byte of the pending match
            if (msrc >= r0) {
                b = my_stage[msrc - r0];
            } else {
                b = cout[(size_t)(msrc >> 2) * 128u + q * 4u + (msrc & 3u)];
            }
            my_stage[o - r0] = (uint8_t)b;
            ++o;
            ++msrc;
            --mrem;
        }
        __syncwarp();
        // rows [r0/4, rend/4): lane l writes column l's word of every row
        const uint32_t rows = (rend - r0) >> 2;
        for (uint32_t i = 0; i < rows; ++i) {
            const uint32_t w = *reinterpret_cast<const uint32_t*>(stage + lane * SSTR + 4 * i);
            reinterpret_cast<uint32_t*>(cout)[(size_t)(r0 / 4 + i) * 32u + lane] = w;
        }
        __syncwarp();
        if (__any_sync(GD_FULL_MASK, err != ST_OK)) break;
    }
    if (err == ST_OK && o != col_bytes) err = ST_CORRUPT;
    return __reduce_max_sync(GD_FULL_MASK, err);
}


}  // namespace lzss
}  // namespace gd
