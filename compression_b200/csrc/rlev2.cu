// rlev2.cu -- RLE v2 (transposed container) decoder for sm_100a.
//
// A block of 4 (or 8) warps owns as many adjacent lane streams of one chunk and copies
// them from the interleaved block into shared memory.  Then, in batches of
// up to RCAP runs per stream:
//   * parse: lane 0 of warp w walks stream w's run boundaries (the only
//     serial part of the format: a run's byte length follows from its first
//     header bytes), recording each run's header offset; then the warp's
//     lanes decode the recorded headers -- kind, length, widths, bit offset
//     of the packed data, base, delta -- into the warp's shared-memory run
//     table, and a warp prefix sum of the lengths gives each run's first
//     value.  After the copy into shared memory the warps
//     of a block never wait on each other, so one warp's walk overlaps the
//     others' expansion;
//   * expand: warp w produces the values of stream w, 32 consecutive values
//     per round, one per lane.  A lane finds its run from a 32-bit map of the
//     run starts inside the round (one shared load and one warp OR-reduce),
//     then computes its value independently: SHORT_REPEAT is the base,
//     DIRECT / PATCHED_BASE unpack a 96-bit big-endian window, fixed DELTA
//     is base + i*delta, and variable DELTA takes a segmented 64-bit warp
//     prefix sum of the unpacked deltas (segments = runs), carried across
//     rounds.  With READ_UNIT a multiple of 32 a round is one contiguous
//     256-byte store;
//   * patch: PATCHED_BASE patch entries are decoded one per lane, placed by a
//     warp prefix sum of their gaps, and OR-ed into the stored values
//     (value = base + (unpacked | patch << width)).
// The grammar and its corrections to the reference are in rlev2.cuh.
#include "rlev2.cuh"

namespace gd {
namespace rlev2 {

constexpr int RCAP = 32;  // runs per stream per batch (small run tables: 8 blocks per SM fit)

// Run tables of one batch (structure of arrays, one row per stream);
// LANES_PER_BLOCK = warps per block = lane streams per block (4 default, 8
// by GD_TUNE_RLEV2_LANES_PER_BLOCK).
// meta = kind | fbw << 2 | flags << 9 | pll << 11 | pw << 16 | cfb << 23;
// aux = delta (DELTA) or the bit offset of the patch list (PATCHED_BASE).
template <int LANES_PER_BLOCK>
struct RunTab {
    uint32_t vs[LANES_PER_BLOCK][RCAP + 1];  // first value of each run; [nr] = end of the batch
    uint32_t pos[LANES_PER_BLOCK][RCAP];     // byte offset of each run's header
    uint32_t meta[LANES_PER_BLOCK][RCAP];
    uint32_t vbit[LANES_PER_BLOCK][RCAP];
    uint64_t base[LANES_PER_BLOCK][RCAP];
    uint64_t aux[LANES_PER_BLOCK][RCAP];
    uint8_t prun[LANES_PER_BLOCK][RCAP];  // PATCHED_BASE runs with patch entries
    uint32_t nr[LANES_PER_BLOCK], npr[LANES_PER_BLOCK];
};

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

template <int LANES_PER_BLOCK>
__global__ void __launch_bounds__(LANES_PER_BLOCK * 32) decode_kernel(
    const uint8_t* __restrict__ data, const uint64_t* __restrict__ col_len, const uint64_t* __restrict__ blk_off,
    uint32_t n_chunks, uint64_t chunk_size, uint32_t ru, uint8_t* __restrict__ out, uint64_t out_n, uint32_t cap,
    uint32_t* __restrict__ status) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ SegTable T_;
    __shared__ uint32_t s_len[32];
    __shared__ uint32_t s_bad;
    __shared__ RunTab<LANES_PER_BLOCK> R;

    const uint32_t lane = lane_id(), wid = threadIdx.x >> 5, tid = threadIdx.x;
    const uint32_t chunk = blockIdx.x / (32 / LANES_PER_BLOCK);
    const uint32_t L0 = (blockIdx.x % (32 / LANES_PER_BLOCK)) * LANES_PER_BLOCK;
    if (chunk >= n_chunks) return;  // block-uniform
    const uint32_t nv = (uint32_t)(chunk_size / 256u);  // values per lane stream
    const uint64_t b0 = blk_off[chunk], b1 = blk_off[chunk + 1];
    const uint8_t* block = data + b0;

    // ---- segment table of the chunk (warp 0) ----
    if (wid == 0) {
        const uint64_t l64 = col_len[32ull * chunk + lane];
        uint32_t bad = (l64 > cap - 32) ? 1u : 0u;  // 16 zeroed + 16 readable bytes follow a stream
        const uint32_t len = bad ? 0u : (uint32_t)l64;
        const uint32_t nw = (len + 3) >> 2;
        uint32_t tot = warp_incl_scan(nw);
        tot = __shfl_sync(GD_FULL_MASK, tot, 31);
        if (b1 < b0 || (uint64_t)tot * 4 > b1 - b0) bad = 1;
        if ((reinterpret_cast<uintptr_t>(block) & 3u) != 0) bad = 1;
        bad = __any_sync(GD_FULL_MASK, bad);
        seg_build(&T_, nw);
        s_len[lane] = len;
        if (lane == 0) s_bad = bad;
    }
    __syncthreads();
    if (s_bad) {
        if (tid == 0 && status) atomicMax(status + chunk, (uint32_t)ST_CORRUPT);
        return;
    }

    // ---- copy this block's 8 lane streams into shared memory ----
    load_lane_streams<LANES_PER_BLOCK>(T_, s_len, block, smem, cap, L0);

    const uint32_t t = L0 + wid;  // the lane stream this warp expands
    const uint8_t* sbuf = smem + wid * cap;
    const uint64_t obase = (uint64_t)chunk * chunk_size;
    const uint64_t want_vals = out_n > obase ? min(chunk_size, out_n - obase) / 8 : 0;  // values of this chunk kept
    uint64_t* outv = reinterpret_cast<uint64_t*>(out + obase);
    const bool ru32 = (ru % 32u) == 0;
    // value e of lane stream t goes to t*ru + (e/ru)*32*ru + e%ru
    auto out_index = [&](uint32_t e) -> uint64_t {
        return (uint64_t)t * ru + (uint64_t)(e / ru) * 32u * ru + (e % ru);
    };

    // parser state: lane 0 of warp w walks stream w, so the walks of a
    // block's streams run on different warps (no divergence between streams,
    // no block barrier: after the copy above each warp runs on its own)
    uint32_t p_pos = 0, p_err = ST_OK;
    const uint32_t plen = s_len[t];
    uint32_t vbeg = 0;  // first value of this warp's current batch
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
                    R.pos[wid][nr++] = p_pos;
                    p_pos += 2u + ((h0 >> 3) & 7u);
                    continue;
                }
                const Skip k = skip_run(sbuf, p_pos, plen);
                if (k.err != ST_OK) {
                    p_err = k.err;
                    break;
                }
                R.pos[wid][nr++] = p_pos;
                p_pos = k.next;
            }
            R.nr[wid] = nr;
            R.npr[wid] = 0;
        }
        __syncwarp();
        // ---- parse 2: decode the recorded headers, one run per lane; run
        // starts are a warp prefix sum of the lengths ----
        const uint32_t nr = R.nr[wid];
        uint32_t perr = ST_OK, carry = vbeg;
        for (uint32_t b0 = 0; b0 < nr; b0 += 32) {
            const uint32_t ri = b0 + lane;
            uint32_t rl = 0;
            if (ri < nr) {
                const Run r = parse_fast(sbuf, R.pos[wid][ri], plen);
                if (r.err != ST_OK) perr = r.err;
                rl = r.len;
                R.meta[wid][ri] = r.kind | (r.fbw << 2) | (r.flags << 9) | (r.pll << 11) | (r.pw << 16) | (r.cfb << 23);
                R.vbit[wid][ri] = r.vbit;
                R.base[wid][ri] = r.base;
                R.aux[wid][ri] = r.kind == 2 ? (uint64_t)r.pbit : r.delta;
                if (r.kind == 2 && r.pll) R.prun[wid][atomicAdd(&R.npr[wid], 1u)] = (uint8_t)ri;
            }
            const uint32_t inc = warp_incl_scan(rl);
            if (ri < nr) R.vs[wid][ri] = carry + inc - rl;
            carry += __shfl_sync(GD_FULL_MASK, inc, 31);
        }
        // the batch's status: a header that runs past the stream, values
        // past the stream's nv, or a stream that ends short of nv values
        const uint32_t pos_now = __shfl_sync(GD_FULL_MASK, p_pos, 0);
        uint32_t berr = max(__reduce_max_sync(GD_FULL_MASK, perr), __shfl_sync(GD_FULL_MASK, p_err, 0));
        if (berr == ST_OK && carry > nv) berr = ST_OVERRUN;
        if (berr == ST_OK && pos_now >= plen && (pos_now != plen || carry != nv)) berr = ST_CORRUPT;
        if (lane == 0) R.vs[wid][nr] = carry;
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
        for (uint32_t rb = vbeg & ~31u; rb < vend; rb += 32) {
            const uint32_t vi = rb + lane;
            const bool act = vi >= vbeg && vi < vend;
            // runs rcur+1 .. rcur+32 cover every run start inside this round
            const int rk = rcur + 1 + (int)lane;
            const uint32_t sk = rk < (int)nr ? R.vs[wid][rk] : 0xffffffffu;
            const uint32_t bm = __reduce_or_sync(GD_FULL_MASK, (sk - rb < 32u) ? (1u << (sk - rb)) : 0u);
            const int rr = rcur + __popc(bm & ((2u << lane) - 1u));
            const uint32_t rrc = rr < 0 ? 0u : (uint32_t)rr;
            const uint32_t meta = R.meta[wid][rrc];
            const uint32_t kind = meta & 3u, fbw = (meta >> 2) & 127u;
            const uint32_t i = vi - R.vs[wid][rrc];  // index of the value inside its run
            const uint64_t base = R.base[wid][rrc];
            uint64_t v = base;
            if (act && (kind == 1u || kind == 2u)) {
                const uint64_t x = extract_msb(sbuf, R.vbit[wid][rrc] + i * fbw, fbw);
                v = kind == 1u ? x : base + x;
            } else if (act && kind == 3u && ((meta >> 9) & 1u)) {
                v = base + (uint64_t)i * R.aux[wid][rrc];
            }
            const bool vdelta = act && kind == 3u && !((meta >> 9) & 1u);
            if (__any_sync(GD_FULL_MASK, vdelta)) {
                // v_0 = base, v_1 = base + delta, v_i = v_{i-1} +- d_{i-2}
                uint64_t sc = 0;
                if (vdelta && i >= 2) sc = extract_msb(sbuf, R.vbit[wid][rrc] + (i - 2) * fbw, fbw);
#pragma unroll
                for (uint32_t o = 1; o < 32; o <<= 1) {
                    const uint64_t n = shfl_up64(sc, o);
                    const int kr = __shfl_up_sync(GD_FULL_MASK, rr, o);
                    if (lane >= o && kr == rr) sc += n;
                }
                if (rr == cr_run) sc += cr_acc;
                if (vdelta) {
                    const uint64_t b1v = base + R.aux[wid][rrc];
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
        }
        __syncwarp();

        // ---- patch entries of this batch's PATCHED_BASE runs ----
        const uint32_t npr = R.npr[wid];
        for (uint32_t q = 0; q < npr; ++q) {
            const uint32_t rp = R.prun[wid][q];
            const uint32_t meta = R.meta[wid][rp];
            const uint32_t fbw = (meta >> 2) & 127u, pll = (meta >> 11) & 31u, pw = (meta >> 16) & 127u,
                           cfb = (meta >> 23) & 127u;
            const uint32_t pbit = (uint32_t)R.aux[wid][rp];
            const uint32_t v0 = R.vs[wid][rp], rlen = R.vs[wid][rp + 1] - v0;
            const uint64_t base = R.base[wid][rp];
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
    if (lane == 0 && werr != ST_OK && status) atomicMax(status + chunk, werr);
}

}  // namespace rlev2
}  // namespace gd

extern "C" gd_status_t gd_rlev2_decode(const uint8_t* d_data, const uint64_t* d_col_len, const uint64_t* d_blk_off,
                                       uint32_t n_chunks, uint64_t chunk_size, uint32_t read_unit,
                                       uint8_t* d_out, uint64_t out_n_bytes, uint32_t max_lane_bytes,
                                       uint32_t* d_status, gd_stream_t stream) {
    if (n_chunks == 0) return GD_OK;
    if (!d_data || !d_col_len || !d_blk_off || !d_out) return GD_ERR_INVALID_ARG;
    if (read_unit == 0) return GD_ERR_UNSUPPORTED;
    if (chunk_size == 0 || chunk_size % (256ull * read_unit) || chunk_size > (1ull << 31)) return GD_ERR_INVALID_ARG;
    if (out_n_bytes > chunk_size * (uint64_t)n_chunks || out_n_bytes <= chunk_size * (uint64_t)(n_chunks - 1))
        return GD_ERR_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(d_out) & 7u) != 0 || out_n_bytes % 8) return GD_ERR_INVALID_ARG;
    using namespace gd::rlev2;
    const uint32_t nv = (uint32_t)(chunk_size / 256u);
    // shared memory per lane stream: the caller's bound on the longest lane
    // stream if given, else the longest a valid stream of nv values can be
    // (a bound above the longest valid stream is clamped: longer lanes are
    // corrupt), plus 16 bytes for the header parser's 24-byte window reads
    const uint32_t cap = (max_lane_bytes ? min(lane_cap(max_lane_bytes), stream_cap(nv)) : stream_cap(nv)) + 16u;
    const int knob = gd_tune_get(GD_TUNE_RLEV2_LANES_PER_BLOCK);
    const int lpb = knob == 8 ? 8 : 4;
    const uint32_t smem = (uint32_t)lpb * cap;
    if (smem > 200 * 1024) return GD_ERR_UNSUPPORTED;  // lane streams must fit in shared memory
    cudaStream_t s = (cudaStream_t)stream;
    // per-chunk status is the max over the chunk's lane streams
    if (d_status && cudaMemsetAsync(d_status, 0, 4ull * n_chunks, s) != cudaSuccess) return GD_ERR_CUDA;
    auto go = [&](auto kern, int lanes) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        kern<<<n_chunks * (32 / lanes), lanes * 32, smem, s>>>(d_data, d_col_len, d_blk_off, n_chunks, chunk_size,
                                                            read_unit, d_out, out_n_bytes, cap, d_status);
    };
    if (lpb == 8) go(decode_kernel<8>, 8);
    else go(decode_kernel<4>, 4);
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}
