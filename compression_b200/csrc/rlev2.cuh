// rlev2.cuh -- RLE v2 (ORC-style integer RLE v2, transposed container)
// decoder for sm_100a.  8-byte values.
//
// Grammar (restated from rlev2::decode_{short_repeat,direct,patched_base,
// delta}, include/rlev2/decoder.h:28-188; the reference GPU decoder_warp,
// decoder_new.h:360-611, decodes the same bytes): the top two header bits
// select SHORT_REPEAT, DIRECT, PATCHED_BASE or DELTA.  Lane t of a chunk owns
// the values t*RU + k*32*RU + j, j < RU.  Corrections to the reference (the
// oracle applies the same): 64-bit patch mask (decoder.h:174 keeps 16 bits),
// the delta accumulation runs len-2 times (decoder.h:117-123 runs len), and
// a PATCHED_BASE base with its top bit set is negative.
//
// The reference decodes a chunk with one decoder warp whose lane t walks lane
// stream t value by value, bit-serially, fed by a reader warp through spin
// queues.  Here every lane stream gets a whole warp:
//   * a block of 8 warps owns 8 adjacent lanes of one chunk; the block copies
//     those 8 streams from the interleaved block into shared memory (row k of
//     the 8 lanes is one contiguous 32-byte sector, located in O(1) through
//     the chunk's segment table);
//   * in each warp, lane 0 parses a run header and broadcasts it, then the 32
//     lanes produce the run's values together: DIRECT / PATCHED_BASE values
//     are unpacked independently (a 96-bit big-endian window per value),
//     PATCHED_BASE patch entries are decoded one per lane and located with a
//     warp prefix sum of their gaps, fixed-delta runs are closed form and
//     variable-delta runs are a 64-bit warp prefix sum;
//   * 32 consecutive values of a lane stream fall in at most two READ_UNIT
//     slices, so each store instruction writes at most two contiguous spans.
#pragma once
#include "interleave.cuh"

namespace gd {
namespace rlev2 {


__device__ __constant__ uint8_t W_DECODE[32] = {1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 13, 14, 15, 16,
                                                17, 18, 19, 20, 21, 22, 23, 24, 26, 28, 30, 32, 40, 48, 56, 64};

__device__ __forceinline__ uint32_t closest_fixed(uint32_t b) {
    if (b <= 1) return 1;
    if (b <= 24) return b;
    if (b <= 26) return 26;
    if (b <= 28) return 28;
    if (b <= 30) return 30;
    if (b <= 32) return 32;
    if (b <= 40) return 40;
    if (b <= 48) return 48;
    if (b <= 56) return 56;
    return 64;
}

// Shared-memory bytes for one lane stream of `nv` values: the largest valid
// stream (64-bit DIRECT runs of 1 value + headers) plus a 16-byte tail that
// unaligned 96-bit reads may touch.
__host__ __device__ constexpr uint32_t stream_cap(uint32_t nv) { return ((nv * 11u + 64u + 15u) & ~15u); }

// Shared-memory bytes reserved for a lane stream of at most `n` bytes.
__host__ __device__ constexpr uint32_t lane_cap(uint32_t n) { return ((n + 15u) & ~15u) + 16u; }

// `w` bits (1..64) starting `bitpos` bits into buf, most significant first
// (the bit order of readLongs, decoder.h:41-72).  buf is 4-byte aligned and
// readable 12 bytes past bitpos/8 rounded down to 4.
__device__ __forceinline__ uint64_t extract_msb(const uint8_t* buf, uint32_t bitpos, uint32_t w) {
    const uint32_t a = bitpos >> 3;
    const uint32_t* p = reinterpret_cast<const uint32_t*>(buf + (a & ~3u));
    const uint32_t s = ((a & 3u) << 3) + (bitpos & 7u);  // 0..31
    const uint32_t w0 = __byte_perm(p[0], 0, 0x0123), w1 = __byte_perm(p[1], 0, 0x0123);
    if (w <= 32) {  // s + w <= 63: two big-endian words, 32-bit arithmetic
        const uint32_t t = __funnelshift_l(w1, w0, s);
        return (uint64_t)(t >> (32u - w));
    }
    const uint32_t w2 = __byte_perm(p[2], 0, 0x0123);
    const uint64_t hi = ((uint64_t)w0 << 32) | w1;
    const uint64_t t = (hi << s) | (((uint64_t)w2 << s) >> 32);
    return w >= 64 ? t : (t >> (64 - w));
}

__device__ __forceinline__ uint64_t shfl64(uint64_t v, int src) {
    const uint32_t lo = __shfl_sync(GD_FULL_MASK, (uint32_t)v, src);
    const uint32_t hi = __shfl_sync(GD_FULL_MASK, (uint32_t)(v >> 32), src);
    return ((uint64_t)hi << 32) | lo;
}

// One parsed run header (filled by lane 0, then broadcast).
struct Run {
    uint32_t kind;   // 0 SR, 1 DIRECT, 2 PATCHED, 3 DELTA
    uint32_t len;    // values
    uint32_t fbw;    // packed width
    uint32_t vbit;   // bit offset of the packed data in the stream
    uint32_t next;   // byte offset of the next header
    uint32_t pw, cfb, pll, pbit;  // patched base: patch width, entry width, entries, list bit offset
    uint32_t flags;  // DELTA: bit0 fixed delta, bit1 subtract
    uint32_t err;
    uint64_t base, delta;
};

__device__ __forceinline__ Run bcast(const Run& r) {
    Run o;
    o.kind = __shfl_sync(GD_FULL_MASK, r.kind, 0);
    o.len = __shfl_sync(GD_FULL_MASK, r.len, 0);
    o.fbw = __shfl_sync(GD_FULL_MASK, r.fbw, 0);
    o.vbit = __shfl_sync(GD_FULL_MASK, r.vbit, 0);
    o.next = __shfl_sync(GD_FULL_MASK, r.next, 0);
    o.pw = __shfl_sync(GD_FULL_MASK, r.pw, 0);
    o.cfb = __shfl_sync(GD_FULL_MASK, r.cfb, 0);
    o.pll = __shfl_sync(GD_FULL_MASK, r.pll, 0);
    o.pbit = __shfl_sync(GD_FULL_MASK, r.pbit, 0);
    o.flags = __shfl_sync(GD_FULL_MASK, r.flags, 0);
    o.err = __shfl_sync(GD_FULL_MASK, r.err, 0);
    o.base = shfl64(r.base, 0);
    o.delta = shfl64(r.delta, 0);
    return o;
}

// Parse the run header at byte `pos` of stream s[0..len) (lane 0 only).
static __device__ Run parse_header(const uint8_t* s, uint32_t pos, uint32_t len) {
    Run r{};
    r.err = ST_OK;
    auto byte = [&](uint32_t& b) -> bool {
        if (pos >= len) return false;
        b = s[pos++];
        return true;
    };
    auto uvarint = [&](uint64_t& v) -> bool {
        uint64_t acc = 0;
        uint32_t sh = 0, b;
        do {
            if (!byte(b)) return false;
            if (sh < 64) acc |= (uint64_t)(b & 0x7fu) << sh;
            sh += 7;
            if (sh > 70) return false;
        } while (b & 0x80u);
        v = acc;
        return true;
    };
    uint32_t first, b;
    if (!byte(first)) {
        r.err = ST_CORRUPT;
        return r;
    }
    r.kind = first >> 6;
    if (r.kind == 0) {  // SHORT_REPEAT, decoder.h:28-39
        const uint32_t nb = ((first >> 3) & 7u) + 1u;
        uint64_t v = 0;
        for (uint32_t i = 0; i < nb; ++i) {
            if (!byte(b)) {
                r.err = ST_CORRUPT;
                return r;
            }
            v = (v << 8) | b;
        }
        r.base = v;
        r.len = (first & 7u) + 3u;
        r.next = pos;
        return r;
    }
    r.fbw = W_DECODE[(first >> 1) & 31u];
    if (!byte(b)) {
        r.err = ST_CORRUPT;
        return r;
    }
    r.len = (((first & 1u) << 8) | b) + 1u;
    if (r.kind == 1) {  // DIRECT, decoder.h:135-142
        r.vbit = pos * 8;
        r.next = pos + (uint32_t)(((uint64_t)r.len * r.fbw + 7) >> 3);
    } else if (r.kind == 2) {  // PATCHED_BASE, decoder.h:144-188
        uint32_t b3, b4;
        if (!byte(b3) || !byte(b4)) {
            r.err = ST_CORRUPT;
            return r;
        }
        const uint32_t bw = ((b3 >> 5) & 7u) + 1u;
        r.pw = W_DECODE[b3 & 31u];
        const uint32_t pgw = ((b4 >> 5) & 7u) + 1u;
        r.pll = b4 & 31u;
        uint64_t bv = 0;
        for (uint32_t i = 0; i < bw; ++i) {
            if (!byte(b)) {
                r.err = ST_CORRUPT;
                return r;
            }
            bv = (bv << 8) | b;
        }
        const uint64_t msb = 1ull << (8 * bw - 1);
        r.base = (bv & msb) ? (uint64_t)(-(int64_t)(bv & ~msb)) : bv;
        r.cfb = closest_fixed(r.pw + pgw);
        r.vbit = pos * 8;
        const uint32_t pstart = pos + (uint32_t)(((uint64_t)r.len * r.fbw + 7) >> 3);
        r.pbit = pstart * 8;
        r.next = pstart + (uint32_t)(((uint64_t)r.pll * r.cfb + 7) >> 3);
    } else {  // DELTA, decoder.h:93-133
        uint64_t ub, zz;
        if (!uvarint(ub) || !uvarint(zz) || r.len < 2) {
            r.err = ST_CORRUPT;
            return r;
        }
        r.base = ub;
        r.delta = (zz >> 1) ^ (0ull - (zz & 1ull));
        const bool fixed = ((first >> 1) & 31u) == 0;
        r.flags = (fixed ? 1u : 0u) | (((int64_t)r.delta > 0) ? 0u : 2u);
        r.vbit = pos * 8;
        r.next = pos + (fixed ? 0u : (uint32_t)(((uint64_t)(r.len - 2) * r.fbw + 7) >> 3));
    }
    if (r.next > len) r.err = ST_CORRUPT;
    return r;
}

// Decode one lane stream (sbuf[0..len), 4-byte aligned, zero padded by 16
// bytes) of nv values with the calling warp.  Lane stream t of a chunk with
// READ_UNIT ru: value e goes to outv[t*ru + (e/ru)*32*ru + e%ru] if that
// index is below want_vals.  Returns a gd status (same on every lane).
static __device__ __noinline__ uint32_t lane_warp(const uint8_t* __restrict__ sbuf, uint32_t len, uint32_t nv, uint32_t t,
                                           uint32_t ru, uint64_t* __restrict__ outv, uint64_t want_vals) {
    const uint32_t lane = lane_id();
    uint32_t err = ST_OK, pos = 0, g = 0;
    while (g < nv) {
        Run r{};
        if (lane == 0) r = parse_header(sbuf, pos, len);
        r = bcast(r);
        if (r.err != ST_OK) {
            err = r.err;
            break;
        }
        if (g + r.len > nv) {
            err = ST_OVERRUN;
            break;
        }
        // patch entries: lane p < pll holds entry p (cumulative index, patch bits)
        uint32_t pidx = 0xffffffffu;
        uint64_t pval = 0;
        if (r.kind == 2) {
            uint32_t gap = 0;
            if (lane < r.pll) {
                const uint64_t e = extract_msb(sbuf, r.pbit + lane * r.cfb, r.cfb);
                gap = (r.pw >= 64) ? 0u : (uint32_t)(e >> r.pw);
                const uint64_t pmask = (r.pw >= 64) ? ~0ull : ((1ull << r.pw) - 1ull);
                pval = (e & pmask) << r.fbw;
            }
            const uint32_t cum = warp_incl_scan(gap);
            if (lane < r.pll) {
                pidx = cum;
                if (cum >= r.len) err = ST_CORRUPT;
            }
            if (__any_sync(GD_FULL_MASK, err != ST_OK)) {
                err = ST_CORRUPT;
                break;
            }
        }
        uint64_t carry = 0;  // DELTA: running sum of unpacked deltas
        for (uint32_t i0 = 0; i0 < r.len; i0 += 32) {
            const uint32_t i = i0 + lane;
            const bool act = i < r.len;
            uint64_t v = 0;
            if (r.kind == 0) {
                v = r.base;
            } else if (r.kind == 1) {
                if (act) v = extract_msb(sbuf, r.vbit + i * r.fbw, r.fbw);
            } else if (r.kind == 2) {
                if (act) v = extract_msb(sbuf, r.vbit + i * r.fbw, r.fbw);
                for (uint32_t p = 0; p < r.pll; ++p) {
                    const uint32_t pi = __shfl_sync(GD_FULL_MASK, pidx, p);
                    const uint64_t pv = shfl64(pval, p);
                    if (pi == i) v |= pv;
                }
                v += r.base;
            } else if (r.flags & 1u) {  // fixed delta: v_i = base + i*delta
                v = r.base + (uint64_t)i * r.delta;
            } else {  // v_0 = base, v_1 = base+delta, v_i = v_{i-1} +- d_{i-2}
                uint64_t d = 0;
                if (act && i >= 2) d = extract_msb(sbuf, r.vbit + (i - 2) * r.fbw, r.fbw);
                uint64_t sc = d;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint64_t n = shfl64(sc, (int)lane - o < 0 ? 0 : (int)lane - o);
                    if (lane >= (uint32_t)o) sc += n;
                }
                const uint64_t acc = carry + sc;
                carry += shfl64(sc, 31);
                const uint64_t b1v = r.base + r.delta;
                v = (i == 0) ? r.base : ((r.flags & 2u) ? b1v - acc : b1v + acc);
            }
            if (act) {
                const uint32_t e = g + i;
                const uint64_t oe = (uint64_t)t * ru + (uint64_t)(e / ru) * 32u * ru + (e % ru);
                if (oe < want_vals) outv[oe] = v;
            }
        }
        pos = r.next;
        g += r.len;
    }
    if (err == ST_OK && pos != len) err = ST_CORRUPT;  // the stream must end with the last run
    return err;
}

}  // namespace rlev2
}  // namespace gd
