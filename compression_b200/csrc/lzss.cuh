// lzss.cuh -- LZSS chunk decoders (the plain kernels in lzss.cu; chunk_warp
// serves the batched decoder in batch.cu).
//
// Grammar (restated from lzss::decompress_func, include/lzss/lzss_gpu2.h:
// 112-325): per column stream, a flag byte then 8 tokens LSB-first; flag 1 =
// one literal byte, flag 0 = little-endian 16-bit v with length (v & 31) + 3
// and offset v >> 5 back into this column's own output.  Column q of a chunk
// owns output bytes 4q + 128k .. +3.  The streams are ranked by descending
// length (col_len sorted, col_map = rank -> column) and 4-byte interleaved.
//
// The reference runs one thread per column with a 2 KiB history array in
// local memory and byte-wise 4-byte-strided stores.  Four decoders here:
//   * chunk_warp (the batch decoder's): a warp per chunk, a lane per column,
//     one output byte per lane and step;
//   * chunk_warp_groups (the default): a warp per chunk, a lane per column,
//     a flag group of tokens per lane and step, output staged per lane in
//     rounds and written as whole rows;
//   * chunk_block_cols: a block per chunk, 8 or 16 lanes per column, the
//     whole chunk staged in shared memory;
//   * chunk_warp_staged: a warp per chunk, a lane per column, the whole chunk
//     staged (3 chunks per SM).
// A match never overlaps its source in the reference encoder's output
// (length <= offset, lzss_gpu2.h:79), but every decoder copies self-
// overlapping matches byte-exactly, as the reference's byte loop does.
#pragma once
#include "interleave.cuh"

namespace gd {
namespace lzss {

// Byte-loop warp decoder (the batch decoder's LZSS path): a warp per chunk,
// a lane per column, one output byte per lane and step.  Each round every
// lane produces 64 bytes (16 output rows) of its column into shared memory,
// then the warp writes those 16 rows (2 KiB contiguous) with coalesced
// stores.  Match sources inside the current round come from shared memory,
// older ones from the already-written output (same SM, ordered by
// __syncwarp).  Inside the batch kernel it measured faster than the group
// decoder below on the mixed batch (19.5 against 21.9 ms, longest-first
// order), although a batch of LZSS chunks alone decodes 1.7x faster with the
// group decoder (5.0 against 8.6 ms): the group decoder's unrolled code added
// to the five decoders' in one kernel overflows the instruction cache
// (warps stalled for instructions 3.5 instead of 1.0 times per issue), which
// slows every codec's tasks.
constexpr uint32_t WARP_RB = 64;             // column bytes per lane per round (16 rows)
constexpr uint32_t WARP_SSTR = WARP_RB + 4;  // 17 words: row reads across columns are conflict-free
constexpr uint32_t WARP_SMEM = (uint32_t)sizeof(SegTable) + 32u * RING_STRIDE + 32u * WARP_SSTR;

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
    const uint32_t rounds = (col_bytes + WARP_RB - 1) / WARP_RB;
    uint8_t* my_stage = stage + q * WARP_SSTR;
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
        const uint32_t r0 = rnd * WARP_RB;
        const uint32_t rend = min(r0 + WARP_RB, col_bytes);
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
            const uint32_t w = *reinterpret_cast<const uint32_t*>(stage + lane * WARP_SSTR + 4 * i);
            reinterpret_cast<uint32_t*>(cout)[(size_t)(r0 / 4 + i) * 32u + lane] = w;
        }
        __syncwarp();
        if (__any_sync(GD_FULL_MASK, err != ST_OK)) break;
    }
    if (err == ST_OK && o != col_bytes) err = ST_CORRUPT;
    return __reduce_max_sync(GD_FULL_MASK, err);
}

// ---------------------------------------------------------------------------
// Group decoder: one warp per chunk, one lane per column, up to NT tokens
// per lane and step (a flag group of 8, or half of one).
//
// The token positions of a group follow from its flag byte alone, so a lane
// loads the group's token bytes together, derives every token's length and
// source with a running sum, loads all match sources before writing
// anything, and appends the tokens through a register holding the column's
// partial word.  The output is produced in rounds of RB column bytes per
// lane: a round's bytes are staged in the lane's own shared-memory slice and
// written out as whole 128-byte rows (the 32 lanes store row k of the chunk
// together: coalesced).  A token may end up to 33 bytes past the round; those
// bytes move to the front of the slice for the next round.  Match sources
// before the round are read back from the output, which this same lane wrote
// (a column's words are stored only by its own lane), so program order makes
// them visible; sources inside the round come from the slice.  With 320-byte
// rounds and a 64-byte input ring a warp holds 14.5 KiB of shared memory, so
// 15 chunks run per SM (3 when the whole 64 KiB output of a chunk is
// staged).  More chunks in flight measured slower: their recent output, which
// the history reads go back to, no longer fits in L2.
// Long (> 8 byte) and self-overlapping (offset < length) matches take a 4-
// or 1-byte loop (byte-exact for every offset >= 1, as the reference's
// byte-wise copy).  The statuses are those of the other decoders: a column
// stops at its first bad token (CORRUPT: stream exhausted, offset 0 or
// before the column start; OVERRUN: past the column end), the chunk reports
// the largest code over its columns.
// ---------------------------------------------------------------------------
constexpr uint32_t GSLACK = 48;  // a round's last token and the 12-byte store window run past RB
__host__ __device__ constexpr uint32_t group_sstr(uint32_t rb) { return rb + GSLACK + 4u; }  // odd word count
// input ring of GR bytes per lane, padded to an odd word count (lanes at
// equal offsets hit distinct banks)
__host__ __device__ constexpr uint32_t group_rstr(uint32_t gr) { return gr + 4u; }
__host__ __device__ constexpr uint32_t group_warp_smem(uint32_t rb, uint32_t gr) {
    return (uint32_t)sizeof(SegTable) + 32u * group_rstr(gr) + 32u * group_sstr(rb);
}

template <uint32_t RB, uint32_t GRING, uint32_t NT = 8>
static __device__ __forceinline__ uint32_t chunk_warp_groups(const uint8_t* __restrict__ block, uint64_t b_len,
                                                            const uint64_t* __restrict__ col_len,
                                                            const uint8_t* __restrict__ col_map, uint64_t chunk_size,
                                                            uint8_t* cout, uint8_t* wsmem) {
    static_assert(RB % 4 == 0 && (group_sstr(RB) / 4) % 2 == 1, "round bytes");
    static_assert(GRING >= 64 && (GRING & (GRING - 1)) == 0, "ring bytes");
    static_assert(NT == 8 || NT == 4, "tokens per step");
    const uint32_t lane = lane_id();
    SegTable* T_ = reinterpret_cast<SegTable*>(wsmem);
    uint8_t* rbuf = wsmem + sizeof(SegTable) + lane * group_rstr(GRING);
    uint32_t* st =
        reinterpret_cast<uint32_t*>(wsmem + sizeof(SegTable) + 32u * group_rstr(GRING) + lane * group_sstr(RB));

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
    if ((reinterpret_cast<uintptr_t>(block) & 3u) != 0) err = ST_CORRUPT;  // words are 4-byte copies
    if ((reinterpret_cast<uintptr_t>(cout) & 3u) != 0) err = ST_INVALID;    // rows are 4-byte stores
    if (chunk_size == 0 || chunk_size % 128 || chunk_size > (1ull << 31)) err = ST_INVALID;
    if (__any_sync(GD_FULL_MASK, err != ST_OK)) return __reduce_max_sync(GD_FULL_MASK, err);
    seg_build(T_, nw);
    const uint32_t ltmask = (1u << lane) - 1u;
    LaneWords lw;
    lw_init(lw, T_, nw);

    const uint32_t col_bytes = (uint32_t)(chunk_size / 32);
    uint32_t* gcol = reinterpret_cast<uint32_t*>(cout) + q;  // column q's word k is gcol[32k]
    uint32_t rd = 0, fl = 0, arrived = 0;  // ring: bytes [rd, arrived) readable, [arrived, fl) in flight
    uint32_t o = 0, acc = 0;               // column bytes produced; the bytes of the partial word o >> 2
    uint32_t flags = 0, ntok = 0;          // the current group's remaining flag bits and tokens
    uint32_t r0 = 0, kr0 = 0;              // the round's first column byte and word

    auto prefetch = [&]() {  // top the ring up (asynchronous 4-byte copies)
        uint32_t n = 0;
        while (lw.k < lw.nw && fl - rd <= GRING - 4u) {
            const uint32_t off = lw_addr(lw, T_, ltmask, lw.k);
            const uint32_t sa = (uint32_t)__cvta_generic_to_shared(rbuf + (fl & (GRING - 1u)));
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(block + off) : "memory");
            fl += 4;
            ++lw.k;
            ++n;
        }
        if (n) asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    auto rb = [&](uint32_t p) -> uint32_t { return rbuf[p & (GRING - 1u)]; };
    // word k of the column: the slice from the round start on, else the output
    auto word = [&](uint32_t k) -> uint32_t { return k >= kr0 ? st[k - kr0] : gcol[(size_t)k * 32u]; };
    auto rd8 = [&](uint32_t sp) -> uint64_t {  // column bytes sp .. sp+7
        const uint32_t k = sp >> 2, sh = (sp & 3u) * 8u;
        const uint32_t w0 = word(k), w1 = word(k + 1u), w2 = word(k + 2u);
        return ((uint64_t)__funnelshift_r(w1, w2, sh) << 32) | __funnelshift_r(w0, w1, sh);
    };
    // append the n (1..8) low bytes of x (zero above them): the partial word
    // and the two words after it are stored (bytes past o are rewritten
    // before anything reads them)
    auto put = [&](uint64_t x, uint32_t n) {
        const uint32_t s = o - r0, sh = (s & 3u) * 8u;
        uint32_t* w = st + (s >> 2);
        const uint64_t v = (uint64_t)acc | (x << sh);
        const uint32_t hi = sh ? (uint32_t)(x >> (64u - sh)) : 0u;
        w[0] = (uint32_t)v;
        w[1] = (uint32_t)(v >> 32);
        w[2] = hi;
        const uint32_t e = (s & 3u) + n;
        acc = e < 4u ? (uint32_t)v : (e < 8u ? (uint32_t)(v >> 32) : hi);
        o += n;
    };
    auto mask = [](uint32_t n) -> uint64_t { return n >= 8u ? ~0ull : ((1ull << (8u * n)) - 1ull); };

    prefetch();
    for (; r0 < col_bytes; r0 += RB, kr0 += RB / 4u) {
        const uint32_t rend = min(r0 + RB, col_bytes);
        for (;;) {
            const bool act = o < rend && err == ST_OK;
            if (!__any_sync(GD_FULL_MASK, act)) break;
            // rings are topped up together once any active lane's is half empty
            if (__any_sync(GD_FULL_MASK, act && fl - rd <= GRING / 2u && lw.k < lw.nw)) prefetch();
            if (!act) continue;
            // a step reads bytes rd .. rd+16 (a flag byte and 8 two-byte tokens)
            if (arrived < fl && arrived < rd + 17u) {
                asm volatile("cp.async.wait_all;\n" ::: "memory");
                arrived = fl;
            }
            if (ntok == 0) {
                if (rd >= len) {
                    err = ST_CORRUPT;
                    continue;
                }
                flags = rb(rd);
                ++rd;
                ntok = 8;
            }
            // the tokens' bytes: token t starts t + (matches before it) bytes after rd
            uint32_t v[NT];
#pragma unroll
            for (uint32_t t = 0; t < NT; ++t) {
                const uint32_t p = rd + t + __popc(~flags & ((1u << t) - 1u));
                v[t] = rb(p) | (rb(p + 1u) << 8);
            }
            // lengths and sources of the tokens that start inside the round;
            // a bad token ends the column
            uint32_t L[NT], src[NT];
            uint32_t p = rd, oo = o, nc = 0;
            bool stop = false;
#pragma unroll
            for (uint32_t t = 0; t < NT; ++t) {
                const bool lit = (flags >> t) & 1u;
                const uint32_t ml = lit ? 1u : (v[t] & 31u) + 3u, off = lit ? 0u : v[t] >> 5;
                const bool live = !stop && t < ntok && oo < rend;
                const bool nobytes = p + (lit ? 0u : 1u) >= len;
                const bool badoff = !lit && (off == 0 || off > oo);
                const bool over = oo + ml > col_bytes;
                if (live && (nobytes || badoff || over)) {
                    err = (nobytes || badoff) ? ST_CORRUPT : ST_OVERRUN;
                    stop = true;
                }
                const bool ok = live && !stop;
                L[t] = ok ? ml : 0u;
                src[t] = oo - off;
                oo += ok ? ml : 0u;
                p += ok ? (lit ? 1u : 2u) : 0u;
                nc += ok ? 1u : 0u;
            }
            // match sources as they are before this group writes anything
            uint64_t x[NT];
#pragma unroll
            for (uint32_t t = 0; t < NT; ++t)
                x[t] = (L[t] && !((flags >> t) & 1u)) ? rd8(src[t]) : (uint64_t)(v[t] & 0xffu);
            const uint32_t o0 = o;
#pragma unroll
            for (uint32_t t = 0; t < NT; ++t) {
                const uint32_t n = L[t];
                if (n == 0) continue;
                const uint32_t sp = src[t], off = o - sp;
                const bool lit = (flags >> t) & 1u;
                if (lit || (n <= 8u && off >= n)) {
                    // a source reaching into this group's output is re-read now
                    const uint64_t y = (!lit && sp + n > o0) ? rd8(sp) : x[t];
                    put(y & mask(n), n);
                } else {
                    // long or self-overlapping match: each piece is read after
                    // the bytes before it are written
                    const uint32_t step = off >= 8u ? 8u : (off >= 4u ? 4u : 1u);
                    for (uint32_t j = 0; j < n; j += step) {
                        const uint32_t m = min(step, n - j);
                        put(rd8(sp + j) & mask(m), m);
                    }
                }
            }
            rd = p;
            flags >>= nc;
            ntok -= nc;
        }
        // the round's rows, then the bytes past it to the front of the slice
        __syncwarp();
        const uint32_t rows = (rend - r0) >> 2;
        for (uint32_t i = 0; i < rows; ++i) gcol[(size_t)(kr0 + i) * 32u] = st[i];
        if (o > rend) {
            const uint32_t cw = (o - rend + 3u) >> 2;
            for (uint32_t i = 0; i < cw; ++i) st[i] = st[rows + i];
        }
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    if (err == ST_OK && o != col_bytes) err = ST_CORRUPT;
    return __reduce_max_sync(GD_FULL_MASK, err);
}

// ---------------------------------------------------------------------------
// Staged decoder: the chunk's whole output lives in shared memory.
//
// The output is staged in its final layout (row k = the k-th 4-byte word of
// all 32 columns, 128 bytes), so column q's words are all in bank q: the 32
// lanes (one column each) never conflict, and a match source anywhere in the
// column's history is a shared-memory read.  A lane handles one flag group
// (8 tokens) per step: token positions follow from the flag byte alone, so
// the 8 tokens' bytes and their match sources (8 bytes each, read before any
// of the group's output is written) are loaded together; then the tokens are
// appended in order through a register holding the column's partial word.
// A source that reaches into the group's own output is re-read when its token
// is appended; long (> 8 byte) and self-overlapping (offset < length)
// matches take a 4- or 1-byte loop (byte-exact for every offset >= 1, as the
// reference's byte-wise copy).  The compressed words of each lane stream are
// prefetched into a per-lane ring with cp.async, well ahead of use.  When
// every column is complete the warp writes the staged rows with 16-byte
// stores.
// ---------------------------------------------------------------------------
constexpr uint32_t STAGE_PAD = 256;  // two rows past the chunk: 8-byte source reads and the carry word
__host__ __device__ constexpr uint32_t staged_smem(uint64_t chunk_size) {
    return (uint32_t)chunk_size + STAGE_PAD + 32u * RING_STRIDE + (uint32_t)sizeof(SegTable);
}

// Per-lane asynchronous ring over the lane's words: bytes [rd, arrived) are
// readable, [arrived, fl) are in flight.
__device__ __forceinline__ void ring_prefetch(LaneRing& r, LaneWords& w, const SegTable* T, const uint8_t* block,
                                              uint32_t ltmask) {
    uint32_t n = 0;
    while (w.k < w.nw && r.fl - r.rd <= (uint32_t)RING - 4u) {
        const uint32_t off = lw_addr(w, T, ltmask, w.k);
        const uint32_t sa = (uint32_t)__cvta_generic_to_shared(r.buf + (r.fl & (RING - 1)));
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(block + off) : "memory");
        r.fl += 4;
        ++w.k;
        ++n;
    }
    if (n) asm volatile("cp.async.commit_group;\n" ::: "memory");
}

static __device__ __noinline__ uint32_t chunk_warp_staged(const uint8_t* __restrict__ block, uint64_t b_len,
                                                         const uint64_t* __restrict__ col_len,
                                                         const uint8_t* __restrict__ col_map, uint64_t chunk_size,
                                                         uint8_t* __restrict__ cout, uint8_t* wsmem) {
    const uint32_t lane = lane_id();
    uint8_t* stage = wsmem;
    uint8_t* ring = wsmem + chunk_size + STAGE_PAD;
    SegTable* T_ = reinterpret_cast<SegTable*>(ring + 32 * RING_STRIDE);

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
    if ((reinterpret_cast<uintptr_t>(block) & 3u) != 0) err = ST_CORRUPT;  // words are 4-byte copies
    if (chunk_size == 0 || chunk_size % 128 || chunk_size > (1ull << 31)) err = ST_INVALID;
    if (__any_sync(GD_FULL_MASK, err != ST_OK)) return __reduce_max_sync(GD_FULL_MASK, err);
    seg_build(T_, nw);
    const uint32_t ltmask = (1u << lane) - 1u;
    LaneWords lw;
    lw_init(lw, T_, nw);
    LaneRing r{ring + lane * RING_STRIDE, 0, 0, len};
    uint32_t arrived = 0;
    ring_prefetch(r, lw, T_, block, ltmask);

    const uint32_t col_bytes = (uint32_t)(chunk_size / 32);
    // column q's word k is stg[32k]
    uint32_t* stg = reinterpret_cast<uint32_t*>(stage) + q;
    uint32_t o = 0, acc = 0;  // column bytes produced; the bytes of the partial word o >> 2

    // append the n (1..8) low bytes of x (zero above them): the partial word,
    // the word after it and the one after that are stored unconditionally
    // (bytes past o are rewritten before anything reads them)
    auto put = [&](uint64_t x, uint32_t n) {
        const uint32_t b = o & 3u, sh = b * 8u;
        uint32_t* w = stg + 32u * (o >> 2);
        const uint64_t v = (uint64_t)acc | (x << sh);
        const uint32_t hi = sh ? (uint32_t)(x >> (64u - sh)) : 0u;
        w[0] = (uint32_t)v;
        w[32] = (uint32_t)(v >> 32);
        w[64] = hi;
        const uint32_t e = b + n;
        acc = e < 4u ? (uint32_t)v : (e < 8u ? (uint32_t)(v >> 32) : hi);
        o += n;
    };
    auto rd8 = [&](uint32_t sp) -> uint64_t {  // column bytes sp .. sp+7
        const uint32_t* w = stg + 32u * (sp >> 2);
        const uint32_t sh = (sp & 3u) * 8u, w1 = w[32];
        return ((uint64_t)__funnelshift_r(w1, w[64], sh) << 32) | __funnelshift_r(w[0], w1, sh);
    };
    auto mask = [](uint32_t n) -> uint64_t { return n >= 8u ? ~0ull : ((1ull << (8u * n)) - 1ull); };

    for (;;) {
        const bool act = (o < col_bytes) && (err == ST_OK);
        if (!__any_sync(GD_FULL_MASK, act)) break;
        // top up every lane's ring together once any active lane is half empty
        const bool low = act && (r.fl - r.rd <= (uint32_t)RING / 2) && (lw.k < lw.nw);
        if (__any_sync(GD_FULL_MASK, low)) ring_prefetch(r, lw, T_, block, ltmask);
        if (!act) continue;
        // the group reads bytes rd .. rd+16
        if (arrived < r.fl && arrived < r.rd + 17u) {
            asm volatile("cp.async.wait_all;\n" ::: "memory");
            arrived = r.fl;
        }
        if (r.rd >= r.len) {
            err = ST_CORRUPT;
            continue;
        }
        const uint32_t flag = ring_byte(r, r.rd);
        // the group's tokens: first and second byte
        uint32_t b0[8], b1[8];
        {
            uint32_t p = r.rd + 1u;
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                b0[t] = ring_byte(r, p);
                b1[t] = ring_byte(r, p + 1u);
                p += 2u - ((flag >> t) & 1u);
            }
        }
        // lengths and sources; a bad token ends the group (and the column)
        uint32_t L[8], src[8];
        uint32_t used = 1;  // group bytes consumed
        {
            uint32_t oo = o, p = r.rd + 1u;
            bool stop = false;
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                const bool lit = (flag >> t) & 1u;
                const uint32_t v = b0[t] | (b1[t] << 8);
                const uint32_t ml = lit ? 1u : (v & 31u) + 3u, off = lit ? 0u : v >> 5;
                const bool live = !stop && oo < col_bytes;
                const bool nobytes = p + (lit ? 0u : 1u) >= r.len;
                const bool badoff = !lit && (off == 0 || off > oo);
                const bool over = oo + ml > col_bytes;
                if (live && (nobytes || badoff || over)) {
                    err = (nobytes || badoff) ? ST_CORRUPT : ST_OVERRUN;
                    stop = true;
                }
                const bool ok = live && !stop;
                L[t] = ok ? ml : 0u;
                src[t] = ok ? oo - off : 0u;
                oo += ok ? ml : 0u;
                used += ok ? (lit ? 1u : 2u) : 0u;
                p += lit ? 1u : 2u;
            }
        }
        // match sources as they are before this group writes anything
        uint64_t x[8];
#pragma unroll
        for (int t = 0; t < 8; ++t) x[t] = (L[t] && !((flag >> t) & 1u)) ? rd8(src[t]) : (uint64_t)b0[t];
        const uint32_t o0 = o;
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            const uint32_t n = L[t];
            if (n == 0) continue;
            const uint32_t sp = src[t], off = o - sp;
            const bool lit = (flag >> t) & 1u;
            if (lit || (n <= 8u && off >= n)) {
                // a source reaching into this group's output is re-read now
                const uint64_t v = (!lit && sp + n > o0) ? rd8(sp) : x[t];
                put(v & mask(n), n);
            } else {
                // long or self-overlapping match: each piece is read after the
                // bytes before it are written
                const uint32_t step = off >= 8u ? 8u : (off >= 4u ? 4u : 1u);
                for (uint32_t j = 0; j < n; j += step) {
                    const uint32_t m = min(step, n - j);
                    put(rd8(sp + j) & mask(m), m);
                }
            }
        }
        r.rd += used;
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    if (err == ST_OK && o != col_bytes) err = ST_CORRUPT;
    err = __reduce_max_sync(GD_FULL_MASK, err);
    __syncwarp();
    if (err == ST_OK) {
        const uint4* s4 = reinterpret_cast<const uint4*>(stage);
        uint4* d4 = reinterpret_cast<uint4*>(cout);
        const uint32_t n16 = (uint32_t)(chunk_size / 16);
        for (uint32_t i = lane; i < n16; i += 32) d4[i] = s4[i];
    }
    return err;
}

// ---------------------------------------------------------------------------
// Column-group decoder: one block per chunk, G = 8 or 16 lanes per column.
//
// The G lanes of a column decode G/8 flag groups per step: lane t takes
// token t (its bytes follow from the flag bytes alone; the second group's
// flag byte sits 17 - popc(first flag) bytes after the first's), the G
// lengths are prefix-summed across the lanes for the output offsets, and
// every token is written at once -- literals and matches whose source lies
// before the step's first output byte (almost all) in one pass, the rest
// (source inside the step's output, offset below the length) in token order
// afterwards.  The
// chunk's output is staged column by column in shared memory (column q at
// q*(col_bytes+4): 8-byte source reads are one funnel shift, and the final
// row-major writes read the 32 columns of a row from 32 different banks).
// Each column's compressed words arrive in a per-column ring by cp.async,
// issued by the column's G lanes half a ring ahead of use.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr uint32_t cols_stride(uint64_t chunk_size) { return (uint32_t)(chunk_size / 32) + 4u; }
__host__ __device__ constexpr uint32_t cols_smem(uint64_t chunk_size) {
    return 32u * cols_stride(chunk_size) + 16u + 32u * RING_STRIDE + (uint32_t)sizeof(SegTable) + 32u * 8u + 16u;
}

// G lanes per column (8: one flag group per step; 16: two, the second's flag
// byte found from the first's).  Must be called by all 32*G threads of the
// block; returns the chunk status.
template <uint32_t G>
static __device__ __forceinline__ uint32_t chunk_block_cols(const uint8_t* __restrict__ block, uint64_t b_len,
                                                           const uint64_t* __restrict__ col_len,
                                                           const uint8_t* __restrict__ col_map,
                                                           uint64_t chunk_size, uint8_t* __restrict__ cout,
                                                           uint8_t* smem) {
    const uint32_t lane = lane_id(), wid = threadIdx.x >> 5;
    const uint32_t cstr = cols_stride(chunk_size);
    uint8_t* stage = smem;
    uint8_t* ring = smem + 32u * cstr + 16u;
    SegTable* T_ = reinterpret_cast<SegTable*>(ring + 32 * RING_STRIDE);
    uint32_t* s_q = reinterpret_cast<uint32_t*>(reinterpret_cast<uint8_t*>(T_) + sizeof(SegTable));
    uint32_t* s_len = s_q + 32;
    uint32_t* s_err = s_len + 32;

    // ---- warp 0: metadata checks and the segment table ----
    if (wid == 0) {
        uint32_t err = ST_OK;
        const uint64_t len64 = col_len[lane];
        const uint32_t len = len64 > 0x3fffffffull ? 0u : (uint32_t)len64;
        if (len64 > 0x3fffffffull) err = ST_CORRUPT;
        const uint32_t q = col_map[lane];
        if (q >= 32) err = ST_CORRUPT;
        uint32_t bits = 0;
#pragma unroll
        for (int o = 0; o < 32; ++o) bits |= 1u << (__shfl_sync(GD_FULL_MASK, q, o) & 31u);
        if (bits != 0xffffffffu) err = ST_CORRUPT;
        const uint32_t nw = (len + 3) >> 2;
        uint32_t tot = warp_incl_scan(nw);
        tot = __shfl_sync(GD_FULL_MASK, tot, 31);
        if ((uint64_t)tot * 4 > b_len) err = ST_CORRUPT;
        if ((reinterpret_cast<uintptr_t>(block) & 3u) != 0) err = ST_CORRUPT;
        if (chunk_size == 0 || chunk_size % 128 || chunk_size > (1ull << 31)) err = ST_INVALID;
        err = __reduce_max_sync(GD_FULL_MASK, err);
        if (err == ST_OK) seg_build(T_, nw);
        s_q[lane] = q & 31u;
        s_len[lane] = len;
        if (lane == 0) *s_err = err;
    }
    __syncthreads();
    if (*s_err != ST_OK) return *s_err;

    static_assert(G == 8 || G == 16, "8 or 16 lanes per column");
    constexpr uint32_t CPW = 32u / G;         // columns per warp
    constexpr uint32_t NWARPS = G;            // warps per block (32 columns)
    constexpr uint32_t GMASK = (1u << G) - 1u;
    constexpr uint32_t NGRP = G / 8u;         // flag groups per step
    const uint32_t sub = lane / G, t = lane % G;
    const uint32_t rank = CPW * wid + sub;
    const uint32_t seg0 = G * sub;  // first lane of this column's group
    const uint32_t cmask = GMASK << seg0;
    const uint32_t q = s_q[rank], len = s_len[rank];
    const uint32_t nw = (len + 3) >> 2;
    const uint32_t col_bytes = (uint32_t)(chunk_size / 32);
    uint8_t* col = stage + q * cstr;
    const uint8_t* rbuf = ring + rank * RING_STRIDE;
    const uint32_t ltmask = (1u << rank) - 1u;
    LaneWords lw;
    lw.k = 0;
    lw.nw = nw;
    lw.j = 0;
    lw_seek_seg(lw, T_, ltmask);
    uint32_t nextk = t;  // this lane copies words t, t+G, t+2G, ... of the stream

    // column state, identical in the column's 8 lanes
    uint32_t rd = 0, o = 0, fl = 0, arrived = 0, err = ST_OK;

    auto prefetch = [&]() {  // top the ring up to 63 words past rd's word
        const uint32_t tgt = min(nw, (rd >> 2) + 63u);
        uint32_t n = 0;
        for (; nextk < tgt; nextk += G) {
            const uint32_t off = lw_addr(lw, T_, ltmask, nextk);
            const uint32_t sa = (uint32_t)__cvta_generic_to_shared(rbuf + ((4u * nextk) & (RING - 1)));
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(block + off) : "memory");
            ++n;
        }
        if (n) asm volatile("cp.async.commit_group;\n" ::: "memory");
        fl = max(fl, 4u * tgt);
    };
    auto rb = [&](uint32_t p) -> uint32_t { return rbuf[p & (RING - 1)]; };
    auto rd8 = [&](uint32_t sp) -> uint64_t {  // column bytes sp .. sp+7
        const uint8_t* a = col + (sp & ~3u);
        const uint32_t* w = reinterpret_cast<const uint32_t*>(a);
        const uint32_t sh = (sp & 3u) * 8u, w1 = w[1];
        return ((uint64_t)__funnelshift_r(w1, w[2], sh) << 32) | __funnelshift_r(w[0], w1, sh);
    };

    prefetch();
    for (;;) {
        const bool act = (o < col_bytes) && (err == ST_OK);
        if (!__any_sync(GD_FULL_MASK, act)) break;
        // rings are topped up together once any active column's is half empty
        if (__any_sync(GD_FULL_MASK, act && fl - rd <= (uint32_t)RING / 2 && fl < 4u * nw) && act) prefetch();
        // a step reads bytes rd .. rd+17*NGRP-1, copied by all G lanes of the column
        const bool wait = act && arrived < fl && arrived < rd + 17u * NGRP;
        if (__any_sync(GD_FULL_MASK, wait)) {
            asm volatile("cp.async.wait_all;\n" ::: "memory");
            __syncwarp();
            arrived = fl;
        }
        uint32_t L = 0, src = 0, ot = 0, lit = 0, code = ST_OK, flag = 0, b0 = 0;
        const uint32_t o0 = o;  // the group's first output byte
        bool exists = false;
        if (act) {
            // flag byte of each group of the step (each follows the previous
            // group's 8 tokens: 17 - popc(flag) bytes after its flag byte)
            uint32_t rds[NGRP], fs[NGRP];
            rds[0] = rd;
            fs[0] = rb(rd);
#pragma unroll
            for (uint32_t gq = 1; gq < NGRP; ++gq) {
                rds[gq] = rds[gq - 1] + 17u - __popc(fs[gq - 1]);
                fs[gq] = rb(rds[gq]);
            }
            const uint32_t gi = t >> 3, tb = t & 7u;
            uint32_t rdg = rds[0];
            flag = fs[0];
#pragma unroll
            for (uint32_t gq = 1; gq < NGRP; ++gq)
                if (gi == gq) {
                    rdg = rds[gq];
                    flag = fs[gq];
                }
            lit = (flag >> tb) & 1u;
            const uint32_t pos = rdg + 1u + tb + __popc(~flag & ((1u << tb) - 1u));
            b0 = rb(pos);
            const uint32_t v = b0 | (rb(pos + 1u) << 8);
            L = lit ? 1u : (v & 31u) + 3u;
            uint32_t inc = L;
#pragma unroll
            for (uint32_t d = 1; d < G; d <<= 1) {
                const uint32_t n = __shfl_up_sync(cmask, inc, d, G);
                if (t >= d) inc += n;
            }
            ot = o + inc - L;
            exists = ot < col_bytes;
            const uint32_t off = lit ? 0u : v >> 5;
            if (exists) {
                if (rdg >= len || pos + (lit ? 0u : 1u) >= len || (!lit && (off == 0 || off > ot)))
                    code = ST_CORRUPT;
                else if (ot + L > col_bytes)
                    code = ST_OVERRUN;
            }
            src = ot - off;
            // the first bad token of the step decides the column's status
            const uint32_t bad = __ballot_sync(cmask, code != ST_OK) >> seg0;
            if (bad) {
                err = __shfl_sync(cmask, code, seg0 + __ffs(bad) - 1u);
            } else {
                const uint32_t total = __shfl_sync(cmask, inc, seg0 + G - 1u);
                o = min(o + total, col_bytes);
                rd = rds[NGRP - 1] + 17u - __popc(fs[NGRP - 1]);
            }
            if (err != ST_OK) exists = false;
        }
        // pass 1: literals and matches whose source lies before the group
        const bool dep = exists && !lit && src + L > o0;
        if (exists && !dep) {
            // the first 8 bytes (a literal: its byte) as predicated stores
            const uint64_t x = lit ? (uint64_t)b0 : rd8(src);
            const uint32_t lo = (uint32_t)x, hi = (uint32_t)(x >> 32);
            uint8_t* d = col + ot;
#pragma unroll
            for (uint32_t i = 0; i < 8; ++i)
                if (i < L) d[i] = (uint8_t)((i < 4 ? lo : hi) >> (8u * (i & 3u)));
            for (uint32_t j = 8; j < L; j += 8) {  // matches longer than 8 bytes
                const uint64_t y = rd8(src + j);
                const uint32_t m = min(8u, L - j);
                for (uint32_t i = 0; i < m; ++i) d[j + i] = (uint8_t)(y >> (8u * i));
            }
        }
        // pass 2: the rest in token order, byte by byte
        if (__any_sync(GD_FULL_MASK, dep)) {
            for (uint32_t tt = 0; tt < G; ++tt) {
                __syncwarp();
                if (dep && t == tt)
                    for (uint32_t j = 0; j < L; ++j) col[ot + j] = col[src + j];
            }
        }
        __syncwarp();
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    if (t == 0 && (err != ST_OK || o != col_bytes)) atomicMax(s_err, err != ST_OK ? err : (uint32_t)ST_CORRUPT);
    __syncthreads();
    const uint32_t e = *s_err;
    if (e == ST_OK) {
        // row k of the chunk = word k of columns 0..31
        const uint32_t rows = col_bytes / 4u;
        uint32_t* o32 = reinterpret_cast<uint32_t*>(cout);
        for (uint32_t k = wid; k < rows; k += NWARPS)
            o32[32u * k + lane] = *reinterpret_cast<const uint32_t*>(stage + lane * cstr + 4u * k);
    }
    return e;
}

}  // namespace lzss
}  // namespace gd
