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
// queues.  Here every lane stream gets a whole warp (decode_stream below):
// lane 0 walks the run boundaries in batches, the warp's lanes decode the
// headers and produce 32 values per round.
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

__device__ __forceinline__ uint64_t shfl_up64(uint64_t v, uint32_t o) {
    const uint32_t lo = __shfl_up_sync(GD_FULL_MASK, (uint32_t)v, o);
    const uint32_t hi = __shfl_up_sync(GD_FULL_MASK, (uint32_t)(v >> 32), o);
    return ((uint64_t)hi << 32) | lo;
}

// W_DECODE as arithmetic: 1..24, then 26, 28, 30, 32, 40, 48, 56, 64
__device__ __forceinline__ uint32_t w_decode(uint32_t c) {
    return c < 24u ? c + 1u : (c < 28u ? 26u + 2u * (c - 24u) : 40u + 8u * (c - 28u));
}

__device__ __forceinline__ uint64_t bswap64(uint64_t x) {
    return ((uint64_t)__byte_perm((uint32_t)x, 0, 0x0123) << 32) | __byte_perm((uint32_t)(x >> 32), 0, 0x0123);
}

// The first n (1..8) bytes of x (x's lowest byte first) as a big-endian number.
__device__ __forceinline__ uint64_t be_bytes(uint64_t x, uint32_t n) { return bswap64(x) >> (64u - 8u * n); }

// parse_header for a stream buffer readable 24 bytes past (pos & ~7): the
// header bytes are taken from one 16-byte window in registers.  SHORT_REPEAT,
// DIRECT and PATCHED_BASE headers (at most 12 bytes) are decoded from the
// window; DELTA headers (varints) use parse_header.
static __device__ __forceinline__ Run parse_fast(const uint8_t* s, uint32_t pos, uint32_t len) {
    Run r{};
    r.err = ST_OK;
    if (pos >= len) {
        r.err = ST_CORRUPT;
        return r;
    }
    const uint64_t* q = reinterpret_cast<const uint64_t*>(s + (pos & ~7u));
    const uint32_t sh = (pos & 7u) * 8u;
    const uint64_t q0 = q[0], q1 = q[1], q2 = q[2];
    const uint64_t lo = sh ? (q0 >> sh) | (q1 << (64u - sh)) : q0;
    const uint64_t hi = sh ? (q1 >> sh) | (q2 << (64u - sh)) : q1;
    const uint32_t b0 = (uint32_t)lo & 0xffu;
    r.kind = b0 >> 6;
    if (r.kind == 3u) return parse_header(s, pos, len);
    if (r.kind == 0u) {  // SHORT_REPEAT: base = bytes 1..nb, big-endian
        const uint32_t nb = ((b0 >> 3) & 7u) + 1u;
        r.base = be_bytes((lo >> 8) | (hi << 56), nb);
        r.len = (b0 & 7u) + 3u;
        r.next = pos + 1u + nb;
    } else {
        r.fbw = w_decode((b0 >> 1) & 31u);
        r.len = (((b0 & 1u) << 8) | ((uint32_t)(lo >> 8) & 0xffu)) + 1u;
        const uint32_t vbytes = (r.len * r.fbw + 7u) >> 3;
        if (r.kind == 1u) {  // DIRECT
            r.vbit = (pos + 2u) * 8u;
            r.next = pos + 2u + vbytes;
        } else {  // PATCHED_BASE: bytes 2, 3, then bw base bytes
            const uint32_t b2 = (uint32_t)(lo >> 16) & 0xffu, b3 = (uint32_t)(lo >> 24) & 0xffu;
            const uint32_t bw = ((b2 >> 5) & 7u) + 1u;
            r.pw = w_decode(b2 & 31u);
            const uint32_t pgw = ((b3 >> 5) & 7u) + 1u;
            r.pll = b3 & 31u;
            const uint64_t bv = be_bytes((lo >> 32) | (hi << 32), bw);
            const uint64_t msb = 1ull << (8u * bw - 1u);
            r.base = (bv & msb) ? (uint64_t)(-(int64_t)(bv & ~msb)) : bv;
            r.cfb = closest_fixed(r.pw + pgw);
            const uint32_t vstart = pos + 4u + bw;
            r.vbit = vstart * 8u;
            const uint32_t pstart = vstart + vbytes;
            r.pbit = pstart * 8u;
            r.next = pstart + ((r.pll * r.cfb + 7u) >> 3);
        }
    }
    if (r.next > len) r.err = ST_CORRUPT;
    return r;
}

// Where the run at byte pos ends and how many values it has, from its
// first 4 header bytes (branch-free for SHORT_REPEAT, DIRECT and
// PATCHED_BASE; DELTA from the ends of its two varints).  This is the only
// serial step of a stream; the headers' fields are decoded afterwards by all
// threads at the recorded positions.  s is readable 24 bytes past
// (pos & ~7) for pos < len.
struct Skip {
    uint32_t next, len, err;
};

// index of the first byte >= i (i <= 15) of the 16 bytes (lo, hi) whose top
// bit is clear (a varint's last byte), 16 if none
__device__ __forceinline__ uint32_t term_from(uint64_t lo, uint64_t hi, uint32_t i) {
    const uint64_t tl = ~lo & 0x8080808080808080ull, th = ~hi & 0x8080808080808080ull;
    const uint64_t ml = i < 8u ? tl & (~0ull << (8u * i)) : 0ull;
    if (ml) return (uint32_t)(__ffsll((long long)ml) - 1) >> 3;
    const uint64_t mh = i <= 8u ? th : th & (~0ull << (8u * (i - 8u)));
    return mh ? 8u + ((uint32_t)(__ffsll((long long)mh) - 1) >> 3) : 16u;
}

static __device__ __forceinline__ Skip skip_run(const uint8_t* s, uint32_t pos, uint32_t len) {
    Skip k;
    k.err = ST_OK;
    k.len = 0;
    k.next = pos;
    if (pos >= len) {
        k.err = ST_CORRUPT;
        return k;
    }
    const uint32_t* q = reinterpret_cast<const uint32_t*>(s + (pos & ~3u));
    const uint32_t w = __funnelshift_r(q[0], q[1], (pos & 3u) * 8u);
    const uint32_t b0 = w & 0xffu, b1 = (w >> 8) & 0xffu, b2 = (w >> 16) & 0xffu, b3 = w >> 24;
    const uint32_t kind = b0 >> 6;
    const uint32_t fbw = w_decode((b0 >> 1) & 31u);
    const uint32_t rl = (((b0 & 1u) << 8) | b1) + 1u;
    if (kind == 3u) {  // DELTA: header, base uvarint, delta svarint, packed deltas
        const uint64_t* q8 = reinterpret_cast<const uint64_t*>(s + (pos & ~7u));
        const uint32_t sh = (pos & 7u) * 8u;
        const uint64_t q0 = q8[0], q1 = q8[1], q2 = q8[2];
        const uint64_t lo = sh ? (q0 >> sh) | (q1 << (64u - sh)) : q0;
        const uint64_t hi = sh ? (q1 >> sh) | (q2 << (64u - sh)) : q1;
        const uint32_t e1 = term_from(lo, hi, 2u);
        const uint32_t e2 = e1 < 15u ? term_from(lo, hi, e1 + 1u) : 16u;
        if (e2 >= 16u || e1 - 2u >= 10u || e2 - e1 - 1u >= 10u) {  // long varints: byte by byte
            const Run r = parse_header(s, pos, len);
            k.err = r.err;
            k.next = r.next;
            k.len = r.len;
            return k;
        }
        const bool fixed = ((b0 >> 1) & 31u) == 0u;
        if (rl < 2u) k.err = ST_CORRUPT;
        k.len = rl;
        k.next = pos + e2 + 1u + (fixed ? 0u : ((rl - 2u) * fbw + 7u) >> 3);
    } else {
        const uint32_t vbytes = (rl * fbw + 7u) >> 3;
        // PATCHED_BASE: base width, patch entry width (closest fixed width of
        // patch width + gap width) and patch count
        const uint32_t bw = (b2 >> 5) + 1u;
        const uint32_t pc = w_decode(b2 & 31u) + (b3 >> 5) + 1u;
        const uint32_t cfb = pc <= 24u ? pc : (pc <= 32u ? (pc + 1u) & ~1u : (pc + 7u) & ~7u);
        const uint32_t npat = 4u + bw + vbytes + (((b3 & 31u) * cfb + 7u) >> 3);
        k.len = kind == 0u ? (b0 & 7u) + 3u : rl;
        k.next = pos + (kind == 0u ? 2u + ((b0 >> 3) & 7u) : (kind == 1u ? 2u + vbytes : npat));
    }
    if (k.next > len) k.err = ST_CORRUPT;
    return k;
}


// ---------------------------------------------------------------------------
// One lane stream decoded by one warp, in batches of up to RCAP runs:
//   * parse 1: lane 0 walks the run boundaries and records only the header
//     positions (the only serial part of the format: a run's byte length
//     follows from its first header bytes);
//   * parse 2: the warp's lanes decode the recorded headers, one run per
//     lane -- kind, length, widths, bit offset of the packed data, base,
//     delta -- into the warp's run table, a warp prefix sum of the lengths
//     gives each run's first value, and the batch is validated;
//   * expand: 32 consecutive values per round, one per lane.  A lane finds
//     its run from a 32-bit map of the run starts inside the round (one
//     shared load and one warp OR-reduce), then computes its value
//     independently: SHORT_REPEAT is the base, DIRECT / PATCHED_BASE unpack a
//     96-bit big-endian window, fixed DELTA is base + i*delta, and variable
//     DELTA takes a segmented 64-bit warp prefix sum of the unpacked deltas
//     (segments = runs), carried across rounds.  With READ_UNIT a multiple of
//     32 a round is one contiguous 256-byte store;
//   * patch: PATCHED_BASE patch entries are decoded one per lane, placed by a
//     warp prefix sum of their gaps, and OR-ed into the stored values
//     (value = base + (unpacked | patch << width)).
// Used by the column decoder (rlev2.cu) and by the batch decoder (batch.cu).
// ---------------------------------------------------------------------------

constexpr int RCAP = 32;  // runs per batch (small run tables: 8 blocks of 4 streams per SM fit)

// The run table of one warp's batch.  meta = kind | fbw << 2 | flags << 9 |
// pll << 11 | pw << 16 | cfb << 23; aux = delta (DELTA) or the bit offset of
// the patch list (PATCHED_BASE).
struct alignas(16) WarpRuns {
    uint64_t base[RCAP];
    uint64_t aux[RCAP];
    uint32_t vs[RCAP + 1];  // first value of each run; [nr] = end of the batch
    uint32_t pos[RCAP];     // byte offset of each run's header
    uint32_t meta[RCAP];
    uint32_t vbit[RCAP];
    uint8_t prun[RCAP];     // PATCHED_BASE runs with patch entries
    uint32_t nr, npr;
};

// sbuf: the lane stream (plen bytes, 4-byte aligned, 16 zero bytes and 16
// more readable bytes after it); nv values; lane stream t of a chunk with
// READ_UNIT ru, values kept below want_vals.  Returns a gd status (the same
// on every lane).
static __device__ __forceinline__ uint32_t decode_stream(const uint8_t* __restrict__ sbuf, uint32_t plen, uint32_t nv,
                                                         uint32_t t, uint32_t ru, uint64_t* __restrict__ outv,
                                                         uint64_t want_vals, WarpRuns& R) {
    const uint32_t lane = lane_id();
    const bool ru32 = (ru % 32u) == 0;
    // value e of lane stream t goes to t*ru + (e/ru)*32*ru + e%ru
    auto out_index = [&](uint32_t e) -> uint64_t {
        return (uint64_t)t * ru + (uint64_t)(e / ru) * 32u * ru + (e % ru);
    };
    uint32_t p_pos = 0, p_err = ST_OK;  // the walk's state (lane 0)
    uint32_t vbeg = 0;                  // first value of the current batch
    uint32_t werr = ST_OK;

    for (;;) {
        // ---- parse 1: run header positions (lane 0) ----
        // Only the positions: a SHORT_REPEAT run's size is in its first byte,
        // the others' in their first 4 (DELTA: the ends of two varints).
        // Run lengths, value starts and all validation come in parse 2.
        if (lane == 0) {
            uint32_t nr = 0;
            while (p_pos < plen && nr < (uint32_t)RCAP) {
                const uint32_t h0 = sbuf[p_pos];
                if (h0 < 64u) {
                    R.pos[nr++] = p_pos;
                    p_pos += 2u + ((h0 >> 3) & 7u);
                    continue;
                }
                const Skip k = skip_run(sbuf, p_pos, plen);
                if (k.err != ST_OK) {
                    p_err = k.err;
                    break;
                }
                R.pos[nr++] = p_pos;
                p_pos = k.next;
            }
            R.nr = nr;
            R.npr = 0;
        }
        __syncwarp();
        // ---- parse 2: decode the recorded headers, one run per lane; run
        // starts are a warp prefix sum of the lengths ----
        const uint32_t nr = R.nr;
        uint32_t perr = ST_OK, carry = vbeg;
        for (uint32_t b0 = 0; b0 < nr; b0 += 32) {
            const uint32_t ri = b0 + lane;
            uint32_t rl = 0;
            if (ri < nr) {
                const Run r = parse_fast(sbuf, R.pos[ri], plen);
                if (r.err != ST_OK) perr = r.err;
                rl = r.len;
                R.meta[ri] = r.kind | (r.fbw << 2) | (r.flags << 9) | (r.pll << 11) | (r.pw << 16) | (r.cfb << 23);
                R.vbit[ri] = r.vbit;
                R.base[ri] = r.base;
                R.aux[ri] = r.kind == 2 ? (uint64_t)r.pbit : r.delta;
                if (r.kind == 2 && r.pll) R.prun[atomicAdd(&R.npr, 1u)] = (uint8_t)ri;
            }
            const uint32_t inc = warp_incl_scan(rl);
            if (ri < nr) R.vs[ri] = carry + inc - rl;
            carry += __shfl_sync(GD_FULL_MASK, inc, 31);
        }
        // the batch's status: a header that runs past the stream, values
        // past the stream's nv, or a stream that ends short of nv values
        const uint32_t pos_now = __shfl_sync(GD_FULL_MASK, p_pos, 0);
        uint32_t berr = max(__reduce_max_sync(GD_FULL_MASK, perr), __shfl_sync(GD_FULL_MASK, p_err, 0));
        if (berr == ST_OK && carry > nv) berr = ST_OVERRUN;
        if (berr == ST_OK && pos_now >= plen && (pos_now != plen || carry != nv)) berr = ST_CORRUPT;
        if (lane == 0) R.vs[nr] = carry;
        __syncwarp();
        if (berr != ST_OK) {
            werr = berr;
            break;
        }

        // ---- expand: values [vbeg, vend) of stream t, 32 per round ----
        const uint32_t vend = carry;
        int rcur = -1;              // run holding the value before this round
        int cr_run = -2;            // run whose delta sum is carried in cr_acc
        uint64_t cr_acc = 0;
        // slice (rb / ru) and offset (rb % ru) of the round, kept incrementally
        uint32_t sl_k = (vbeg & ~31u) / ru, sl_j = (vbeg & ~31u) % ru;
        for (uint32_t rb = vbeg & ~31u; rb < vend;) {
            // ---- fast path: rounds inside one run (warp-uniform) ----
            // The run holding value rb is rcur, or rcur + 1 when a run starts
            // exactly at rb.  While whole rounds lie inside it, every lane
            // decodes the same run with its fields held in registers: no run
            // search, one kind, no divergence.
            {
                const int nx = rcur + 1;
                const int r0 = (nx < (int)nr && R.vs[nx] == rb) ? nx : rcur;
                const uint32_t rend = r0 >= 0 ? min(R.vs[r0 + 1], vend) : 0u;
                if (r0 >= 0 && rb >= vbeg && rb + 32u <= rend) {
                    const uint32_t meta = R.meta[r0];
                    const uint32_t kind = meta & 3u, fbw = (meta >> 2) & 127u;
                    const uint32_t v0 = R.vs[r0];
                    const uint64_t base = R.base[r0], aux = R.aux[r0];
                    const uint32_t vbit = R.vbit[r0];
                    const bool fixed = ((meta >> 9) & 1u) != 0, sub = ((meta >> 10) & 1u) != 0;
                    if (kind == 3u && !fixed && r0 != cr_run) cr_acc = 0;
                    // bit-packed kinds: two rounds per iteration, so that the
                    // two unpack chains overlap
                    if (ru32 && (kind == 1u || kind == 2u)) {
                        for (; rb + 64u <= rend; rb += 64) {
                            const uint32_t i = rb + lane - v0;
                            const uint64_t xa = extract_msb(sbuf, vbit + i * fbw, fbw);
                            const uint64_t xb = extract_msb(sbuf, vbit + (i + 32u) * fbw, fbw);
                            const uint64_t oa = (uint64_t)t * ru + (uint64_t)sl_k * 32u * ru + sl_j + lane;
                            sl_j += 32;
                            if (sl_j >= ru) {
                                sl_j -= ru;
                                ++sl_k;
                            }
                            const uint64_t ob = (uint64_t)t * ru + (uint64_t)sl_k * 32u * ru + sl_j + lane;
                            sl_j += 32;
                            if (sl_j >= ru) {
                                sl_j -= ru;
                                ++sl_k;
                            }
                            if (oa < want_vals) outv[oa] = kind == 1u ? xa : base + xa;
                            if (ob < want_vals) outv[ob] = kind == 1u ? xb : base + xb;
                        }
                    }
                    while (rb + 32u <= rend) {
                        const uint32_t i = rb + lane - v0;  // index of this lane's value in the run
                        uint64_t v = base;
                        if (kind == 1u || kind == 2u) {
                            const uint64_t x = extract_msb(sbuf, vbit + i * fbw, fbw);
                            v = kind == 1u ? x : base + x;
                        } else if (kind == 3u) {
                            if (fixed) {
                                v = base + (uint64_t)i * aux;
                            } else {
                                // v_0 = base, v_1 = base + delta, v_i = v_{i-1} +- d_{i-2}
                                uint64_t sc = i >= 2 ? extract_msb(sbuf, vbit + (i - 2) * fbw, fbw) : 0ull;
#pragma unroll
                                for (uint32_t o = 1; o < 32; o <<= 1) {
                                    const uint64_t n = shfl_up64(sc, o);
                                    if (lane >= o) sc += n;
                                }
                                sc += cr_acc;
                                const uint64_t b1v = base + aux;
                                v = (i == 0) ? base : (sub ? b1v - sc : b1v + sc);
                                cr_acc = shfl64(sc, 31);
                            }
                        }
                        const uint64_t oe = ru32 ? (uint64_t)t * ru + (uint64_t)sl_k * 32u * ru + sl_j + lane
                                                 : out_index(rb + lane);
                        if (oe < want_vals) outv[oe] = v;
                        sl_j += 32;
                        if (sl_j >= ru) {
                            sl_j -= ru;
                            ++sl_k;
                        }
                        rb += 32;
                    }
                    rcur = r0;
                    cr_run = r0;
                    continue;
                }
            }
            const uint32_t vi = rb + lane;
            const bool act = vi >= vbeg && vi < vend;
            // runs rcur+1 .. rcur+32 cover every run start inside this round
            const int rk = rcur + 1 + (int)lane;
            const uint32_t sk = rk < (int)nr ? R.vs[rk] : 0xffffffffu;
            const uint32_t bm = __reduce_or_sync(GD_FULL_MASK, (sk - rb < 32u) ? (1u << (sk - rb)) : 0u);
            const int rr = rcur + __popc(bm & ((2u << lane) - 1u));
            const uint32_t rrc = rr < 0 ? 0u : (uint32_t)rr;
            const uint32_t meta = R.meta[rrc];
            const uint32_t kind = meta & 3u, fbw = (meta >> 2) & 127u;
            const uint32_t i = vi - R.vs[rrc];  // index of the value inside its run
            const uint64_t base = R.base[rrc];
            uint64_t v = base;
            if (act && (kind == 1u || kind == 2u)) {
                const uint64_t x = extract_msb(sbuf, R.vbit[rrc] + i * fbw, fbw);
                v = kind == 1u ? x : base + x;
            } else if (act && kind == 3u && ((meta >> 9) & 1u)) {
                v = base + (uint64_t)i * R.aux[rrc];
            }
            const bool vdelta = act && kind == 3u && !((meta >> 9) & 1u);
            if (__any_sync(GD_FULL_MASK, vdelta)) {
                // v_0 = base, v_1 = base + delta, v_i = v_{i-1} +- d_{i-2}
                uint64_t sc = 0;
                if (vdelta && i >= 2) sc = extract_msb(sbuf, R.vbit[rrc] + (i - 2) * fbw, fbw);
#pragma unroll
                for (uint32_t o = 1; o < 32; o <<= 1) {
                    const uint64_t n = shfl_up64(sc, o);
                    const int kr = __shfl_up_sync(GD_FULL_MASK, rr, o);
                    if (lane >= o && kr == rr) sc += n;
                }
                if (rr == cr_run) sc += cr_acc;
                if (vdelta) {
                    const uint64_t b1v = base + R.aux[rrc];
                    v = (i == 0) ? base : (((meta >> 10) & 1u) ? b1v - sc : b1v + sc);
                }
                cr_acc = shfl64(sc, 31);
            }
            rcur = __shfl_sync(GD_FULL_MASK, rr, 31);
            cr_run = rcur;
            if (act) {
                const uint64_t oe = ru32 ? (uint64_t)t * ru + (uint64_t)sl_k * 32u * ru + sl_j + lane : out_index(vi);
                if (oe < want_vals) outv[oe] = v;
            }
            sl_j += 32;
            if (sl_j >= ru) {
                sl_j -= ru;
                ++sl_k;
            }
            rb += 32;
        }
        __syncwarp();

        // ---- patch entries of this batch's PATCHED_BASE runs ----
        const uint32_t npr = R.npr;
        for (uint32_t q = 0; q < npr; ++q) {
            const uint32_t rp = R.prun[q];
            const uint32_t meta = R.meta[rp];
            const uint32_t fbw = (meta >> 2) & 127u, pll = (meta >> 11) & 31u, pw = (meta >> 16) & 127u,
                           cfb = (meta >> 23) & 127u;
            const uint32_t pbit = (uint32_t)R.aux[rp];
            const uint32_t v0 = R.vs[rp], rlen = R.vs[rp + 1] - v0;
            const uint64_t base = R.base[rp];
            uint32_t gap = 0;
            uint64_t P = 0;
            if (lane < pll) {
                const uint64_t e = extract_msb(sbuf, pbit + lane * cfb, cfb);
                gap = (pw >= 64) ? 0u : (uint32_t)(e >> pw);
                const uint64_t pmask = (pw >= 64) ? ~0ull : ((1ull << pw) - 1ull);
                P = (fbw >= 64) ? 0ull : ((e & pmask) << fbw);
            }
            const uint32_t cum = warp_incl_scan(gap);  // index of entry `lane` inside the run
            // entries that land on the same value are OR-ed together
#pragma unroll
            for (uint32_t o = 1; o < 32; o <<= 1) {
                const uint64_t n = shfl_up64(P, o);
                const uint32_t c2 = __shfl_up_sync(GD_FULL_MASK, cum, o);
                if (lane >= o && c2 == cum) P |= n;
            }
            const uint32_t cnext = __shfl_down_sync(GD_FULL_MASK, cum, 1);
            const bool last = lane < pll && (lane + 1 == pll || cnext != cum);
            if (__any_sync(GD_FULL_MASK, lane < pll && cum >= rlen)) {
                werr = ST_CORRUPT;
                continue;
            }
            if (last) {
                const uint64_t oe = out_index(v0 + cum);
                if (oe < want_vals) outv[oe] = ((outv[oe] - base) | P) + base;
            }
        }
        vbeg = vend;
        __syncwarp();  // the next batch rewrites this warp's run tables
        if (pos_now >= plen) break;  // the stream is consumed (and held exactly nv values)
    }
    return werr;
}

}  // namespace rlev2
}  // namespace gd
