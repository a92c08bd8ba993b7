// rlev1.cuh -- RLE v1 (ORC-style integer RLE v1) decoder for sm_100a.
//
// Grammar (restated from decoder_warp, include/rle_v1/decoder.h:278-423):
// int8 header h; h < 0: -h literal values, each an unsigned LEB128 varint;
// h >= 0: a run of h+3 values, int8 delta then varint base, v_i = base+i*delta.
// Lane t of a chunk owns elements (i / wil)*32*wil + t*wil + i % wil,
// wil = COMP_COL_LEN / sizeof(T); a lane stream ends once it has produced
// chunk_size/32 bytes (decoder.h:283,291).
//
// The reference pairs a reader warp and a decoder warp per chunk (spin
// queues, one byte fetched per funnel-shift call, one scalar store per
// value).  Here every lane stream gets a whole warp (same block loader as
// RLE v2: 8 adjacent lane streams per block, copied with fully used 32-byte
// row sectors):
//   * runs are closed form: lane i writes base + i*delta;
//   * a literal group is decoded 32 values at a time: the lanes load a
//     128-byte window, ballot the varint terminators (bytes < 0x80), and lane
//     j finds the j-th terminator (the mask quarter by comparison with the
//     quarters' prefix counts, then one select), so every lane knows where
//     its varint starts and ends and decodes it alone (32-bit values: one
//     funnel-shifted word and a fifth byte, compacted with masks).
#pragma once
#include "interleave.cuh"

namespace gd {
namespace rlev1 {


// Largest lane stream for nv values: literal varints of up to 10 bytes plus
// one header per 127 values; +128 tail for terminator windows.
__host__ __device__ constexpr uint32_t stream_cap(uint32_t nv, uint32_t eb) {
    return (((eb == 8 ? 10u : 5u) * nv + nv / 127u + 64u + 15u) & ~15u) + 144u;
}

// Shared-memory bytes reserved for a lane stream of at most `n` bytes.
__host__ __device__ constexpr uint32_t lane_cap(uint32_t n) { return ((n + 15u) & ~15u) + 144u; }

// Decode one lane stream (sbuf[0..len), readable 144 bytes past len) of nv
// elements of type T with the calling warp.  Lane stream t with wil = values
// per lane slice: element e goes to outv[(e/wil)*32*wil + t*wil + e%wil] if
// that index is below want.  Returns a gd status (same on every lane).
template <typename T>
static __device__ __noinline__ uint32_t lane_warp(const uint8_t* __restrict__ sbuf, uint32_t len, uint32_t nv, uint32_t t,
                                           uint32_t wil, T* __restrict__ outv, uint64_t want) {
    const uint32_t lane = lane_id();
    // wil a power of two (COMP_COL_LEN / sizeof(T) always is in the
    // reference's configurations): shifts instead of a division per value
    const bool pow2 = (wil & (wil - 1u)) == 0u;
    const uint32_t wsh = __ffs(wil) - 1u;
    // a chunk holds at most 2^31 bytes, so element indices fit in 32 bits
    const uint32_t want32 = want < 0xffffffffull ? (uint32_t)want : 0xffffffffu;
    const uint32_t tw = t << wsh;
    auto put = [&](uint32_t e, T v) {
        const uint32_t oe = pow2 ? ((e >> wsh) << (wsh + 5u)) + tw + (e & (wil - 1u))
                                 : (e / wil) * 32u * wil + t * wil + (e % wil);
        if (oe < want32) outv[oe] = v;
    };
    uint32_t err = ST_OK, pos = 0, g = 0;
    while (g < nv) {
        // ---- header: every lane parses it (shared-memory broadcast reads),
        // so nothing needs to be shuffled ----
        uint32_t kind = 0, cnt = 0, next = 0, e = ST_OK;
        uint64_t base = 0, delta = 0;
        {
            uint32_t p = pos;
            if (p >= len) {
                e = ST_CORRUPT;
            } else {
                const uint32_t h = sbuf[p++];
                if (h & 0x80u) {
                    kind = 1;
                    cnt = 256u - h;
                } else if (p >= len) {
                    e = ST_CORRUPT;
                } else {
                    kind = 0;
                    cnt = h + 3u;
                    delta = (uint64_t)(int64_t)(int8_t)sbuf[p++];
                    uint32_t sh = 0, b;
                    do {
                        if (p >= len || sh > 63) {
                            e = ST_CORRUPT;
                            break;
                        }
                        b = sbuf[p++];
                        base |= (uint64_t)(b & 0x7fu) << sh;
                        sh += 7;
                    } while (b & 0x80u);
                    if (sizeof(T) == 4) base &= 0xffffffffull;
                }
            }
            next = p;
        }
        if (e != ST_OK) {
            err = e;
            break;
        }
        if (g + cnt > nv) {
            err = ST_OVERRUN;
            break;
        }
        if (kind == 0) {  // run: closed form (in T's width: the low bits of base + i*delta)
            for (uint32_t i = lane; i < cnt; i += 32) put(g + i, (T)base + (T)i * (T)delta);
            g += cnt;
            pos = next;
            continue;
        }
        // literal group: cnt varints starting at `next`
        uint32_t p = next, rem = cnt;
        while (rem) {
            uint32_t m[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint32_t bpos = p + 32u * q + lane;
                const bool term = (bpos < len) && !(sbuf[bpos] & 0x80u);
                m[q] = __ballot_sync(GD_FULL_MASK, term);
            }
            const uint32_t c0 = __popc(m[0]), c01 = c0 + __popc(m[1]), c012 = c01 + __popc(m[2]);
            const uint32_t nterm = c012 + __popc(m[3]);
            if (nterm == 0) {  // no varint ends within 128 bytes (or the stream ran out)
                err = ST_CORRUPT;
                break;
            }
            const uint32_t take = min(min(rem, nterm), 32u);
            // lane j's varint ends at the j-th terminator: its 32-bit quarter
            // of the mask by comparison, then one select within it
            uint32_t end = 0;
            if (lane < take) {
                const uint32_t q = (lane >= c0) + (lane >= c01) + (lane >= c012);
                const uint32_t mq = q == 0 ? m[0] : (q == 1 ? m[1] : (q == 2 ? m[2] : m[3]));
                const uint32_t nq = lane - (q == 0 ? 0u : (q == 1 ? c0 : (q == 2 ? c01 : c012)));
                end = 32u * q + __fns(mq, 0, (int)nq + 1);
            }
            const uint32_t prev = __shfl_up_sync(GD_FULL_MASK, end, 1);  // the previous varint's last byte
            if (lane < take) {
                const uint32_t beg = lane ? prev + 1 : 0;
                uint64_t v = 0;
                if constexpr (sizeof(T) == 4) {
                    // a 32-bit value takes the varint's first 5 bytes: the
                    // first 4 by one funnel-shifted word, 7 bits apiece
                    const uint32_t a = p + beg, n = end - beg + 1;
                    const uint32_t* wp = reinterpret_cast<const uint32_t*>(sbuf + (a & ~3u));
                    uint32_t lo = __funnelshift_r(wp[0], wp[1], 8u * (a & 3u));
                    if (n < 4) lo &= (1u << (8u * n)) - 1u;
                    const uint32_t hi = n >= 5 ? (uint32_t)sbuf[a + 4] : 0u;
                    v = (lo & 0x7fu) | ((lo >> 1) & 0x3f80u) | ((lo >> 2) & 0x1fc000u) | ((lo >> 3) & 0xfe00000u) |
                        (hi << 28);
                } else {
                    uint32_t sh = 0;
                    for (uint32_t k = beg; k <= end; ++k, sh += 7)
                        if (sh < 64) v |= (uint64_t)(sbuf[p + k] & 0x7fu) << sh;
                }
                put(g + lane, (T)v);
            }
            p += __shfl_sync(GD_FULL_MASK, end, take - 1) + 1;
            g += take;
            rem -= take;
        }
        if (err != ST_OK) break;
        pos = p;
    }
    return err;
}

}  // namespace rlev1
}  // namespace gd
