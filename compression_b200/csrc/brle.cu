// brle.cu -- byte-RLE (brle.h container) decoder for sm_100a.
//
// Format (restated from brle::decode, include/brle/brle.h:76-97): a chunk is
// a sequence of tokens; control byte c > 127 is followed by c-127 literal
// bytes, c <= 127 by one byte repeated c+3 times.  Chunk c's tokens occupy
// data[ptr[c] .. ptr[c+1]) and expand to out[c*chunk_size ..].
//
// The reference decodes one chunk per thread (1024 threads on the whole GPU
// for a 256 MiB column).  Here one 256-thread block decodes a chunk, 9 KiB of
// compressed bytes (a tile) at a time:
//   1. The tile (+ a 160-byte halo for tokens that run past it) is staged in
//      shared memory with 16-byte loads.
//   2. Token starts form a chain (each token is 2..129 bytes).  Thread t owns
//      a 36-byte segment and computes, by one backward pass over its bytes,
//      where the chain leaves the segment for every entry offset (an exit
//      table).
//   3. Warp w owns a region of 32 segments.  Lane l follows the chain
//      through the region from entry offset l of its first segment, one table
//      lookup per segment, recording the entry of every segment.  All 32
//      possible region entries are thus resolved in parallel.
//   4. One thread links the 8 regions (8 lookups; an entry that a long
//      literal carried past a region's first segment is walked through the
//      segment tables instead), and every segment learns its true entry.
//   5. Each thread walks its segment's tokens: output bytes, token count and
//      validation; a block scan places every token, and each thread writes
//      its tokens into the tile's token list (output offset, position,
//      control byte, run byte).
//   6. Expansion: the tile's output is cut into 64-byte slices dealt round
//      robin to all 256 threads.  A thread finds the token covering its slice
//      in a slice -> token index written with the list (a binary search of
//      the list for tiles with more output than the index holds), builds each aligned
//      16-byte vector by merging the pieces of the tokens that cover it (a run
//      piece is a broadcast byte, a literal piece an unaligned 16-byte read
//      of the staged tile), and stores it with one 16-byte store.  The few
//      vectors shared with the neighbouring tile are stored bytewise.
// Every read is bounded by the chunk's compressed length and every write by
// its output size; a malformed chunk gets GD_ERR_CORRUPT / GD_ERR_OVERRUN.
#include "gd_common.cuh"

namespace gd {
namespace brle {

constexpr int NT = 256;
constexpr int NWARP = NT / 32;
// compressed bytes per thread segment: 36, not 32, so that the 32 lanes of a
// warp, each in its own segment at the same offset, address 32 different
// shared-memory banks (a 32-byte stride puts 8 lanes on every bank)
constexpr int SEG = 36;
constexpr int REG = 32 * SEG;    // bytes per warp region
constexpr int TILE = NT * SEG;   // compressed bytes per tile
constexpr int HALO = 160;        // a token starting in the tile reads <= 128 more bytes
constexpr uint32_t NONE = 0xffffffffu;
constexpr uint32_t FALLBACK = 0x100u;
constexpr uint32_t MAXTOK = TILE / 2;  // a token is >= 2 bytes
// dynamic shared memory: staged tile (16 B front pad, alignment shift, tail
// pad for unaligned 16-byte reads), exit tables, token list (which also holds
// the region chains before the list is built)
constexpr uint32_t OFF_TILE = 0;
constexpr uint32_t TILE_BYTES = 16 + 16 + TILE + HALO + 32;
constexpr uint32_t OFF_TBL = (TILE_BYTES + 15u) & ~15u;
constexpr uint32_t OFF_LIST = OFF_TBL + TILE;
constexpr uint32_t SMEM = OFF_LIST + MAXTOK * 8;
static_assert(NWARP * 32 * 32 * 2 <= MAXTOK * 8, "region chains must fit in the token list space");
constexpr uint32_t SLICE_CAP = TILE / 2;  // 64-byte slices indexed per tile (u16 entries in the exit tables)

__device__ __forceinline__ uint32_t tok_in(uint32_t c) { return c > 127u ? c - 126u : 2u; }
__device__ __forceinline__ uint32_t tok_out(uint32_t c) { return c > 127u ? c - 127u : c + 3u; }

// 16 bytes at any shared-memory address p (8-byte aligned reads p&~7 .. +24).
__device__ __forceinline__ void lds16_unaligned(const uint8_t* p, uint64_t& lo, uint64_t& hi) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const uint64_t* q = reinterpret_cast<const uint64_t*>(a & ~(uintptr_t)7);
    const uint32_t sh = (uint32_t)(a & 7u) * 8u;
    const uint64_t q0 = q[0], q1 = q[1], q2 = q[2];
    lo = sh ? (q0 >> sh) | (q1 << (64u - sh)) : q0;
    hi = sh ? (q1 >> sh) | (q2 << (64u - sh)) : q1;
}

__global__ void __launch_bounds__(NT, 4) decode_kernel(const uint8_t* __restrict__ data,
                                                       const uint64_t* __restrict__ ptr, uint32_t n_chunks,
                                                       uint64_t chunk_size, uint8_t* __restrict__ out,
                                                       uint64_t out_n, uint32_t* __restrict__ status) {
    extern __shared__ __align__(16) uint8_t s_dyn[];
    uint8_t* s_tbl = s_dyn + OFF_TBL;
    uint2* s_list = reinterpret_cast<uint2*>(s_dyn + OFF_LIST);
    uint16_t* s_chain = reinterpret_cast<uint16_t*>(s_dyn + OFF_LIST);  // [warp][segment][lane]
    __shared__ uint32_t s_entry[NT];
    __shared__ uint16_t s_rx[NWARP][32];
    __shared__ uint32_t s_rentry[NWARP];
    __shared__ uint64_t s_scan[NWARP + 1];
    __shared__ uint32_t s_carry;

    const uint32_t tid = threadIdx.x, lane = tid & 31u, wid = tid >> 5;
    for (uint32_t chunk = blockIdx.x; chunk < n_chunks; chunk += gridDim.x) {
        const uint64_t beg = ptr[chunk], end = ptr[chunk + 1];
        const uint64_t obase = (uint64_t)chunk * chunk_size;
        uint32_t err = ST_OK;
        if (end < beg || end - beg > 0x7fffffffull || obase >= out_n) err = ST_CORRUPT;
        const uint32_t clen = err ? 0u : (uint32_t)(end - beg);
        const uint32_t want = err ? 0u : (uint32_t)(out_n - obase < chunk_size ? out_n - obase : chunk_size);
        const uint8_t* src = data + beg;
        uint8_t* dst = out + obase;
        const bool aligned16 = ((reinterpret_cast<uintptr_t>(dst) & 15u) == 0);

        uint32_t carry = 0;  // chunk-relative position of the next token start
        uint32_t opos = 0;   // output bytes placed so far

        for (uint32_t t0 = 0; t0 < clen && err == ST_OK; t0 += TILE) {
            // positions below are tile-relative; cl = chunk end in tile coordinates
            const uint32_t cl = clen - t0;
            // ---- 1. stage compressed bytes [t0, min(clen, t0+TILE+HALO)) ----
            // Tile byte i lives at tb[i], tb = s_dyn + 16 + (global address mod
            // 16), so aligned 16-byte global words land on aligned shared words.
            const uint32_t n_ld = min(cl, (uint32_t)(TILE + HALO));
            const uint8_t* g = src + t0;
            const uint32_t sh = (uint32_t)(reinterpret_cast<uintptr_t>(g) & 15u);
            uint8_t* tb = s_dyn + OFF_TILE + 16 + sh;
            {
                uint32_t head = (16u - sh) & 15u;
                if (head > n_ld) head = n_ld;
                if (tid < head) tb[tid] = g[tid];
                const uint32_t nv = (n_ld - head) >> 4;
                const uint4* gv = reinterpret_cast<const uint4*>(g + head);
                uint4* sv = reinterpret_cast<uint4*>(tb + head);
                for (uint32_t i = tid; i < nv; i += NT) sv[i] = __ldg(gv + i);
                for (uint32_t i = head + 16 * nv + tid; i < n_ld; i += NT) tb[i] = g[i];
            }
            __syncthreads();

            // ---- 2. exit table of this thread's segment ----
            // s_tbl[p] = (chain exit - S) when the chain passes p in [S, lim);
            // an exit is the first chain position >= lim (<= SEG - 1 + 129).
            const uint32_t S = SEG * tid;
            const uint32_t lim = min(S + SEG, cl);
            if (S < cl) {
                for (int32_t p = (int32_t)lim - 1; p >= (int32_t)S; --p) {
                    const uint32_t n = (uint32_t)p + tok_in(tb[p]);
                    s_tbl[p] = (n >= lim) ? (uint8_t)(n - S) : s_tbl[n];
                }
            }
            __syncthreads();

            // ---- 3. chains through this warp's region, one per entry offset ----
            {
                const uint32_t R = REG * wid;
                uint32_t e = R + lane;
                uint16_t* ch = s_chain + wid * 32 * 32;
#pragma unroll 4
                for (uint32_t j = 0; j < 32; ++j) {
                    const uint32_t Sj = R + SEG * j;
                    const uint32_t lj = min(Sj + SEG, cl);
                    uint16_t rec = 0xffff;
                    if (e < lj) {  // e >= Sj always holds here
                        rec = (uint16_t)e;
                        e = Sj + s_tbl[e];
                    }
                    ch[j * 32 + lane] = rec;
                }
                s_rx[wid][lane] = (uint16_t)min(e, 0xffffu);
            }
            __syncthreads();

            // ---- 4. link the regions ----
            if (tid == 0) {
                uint32_t e = carry - t0;  // < 129: the previous tile's last token ends here
                for (uint32_t w = 0; w < (uint32_t)NWARP; ++w) {
                    const uint32_t R = REG * w;
                    if (R >= cl || e >= R + REG) {
                        s_rentry[w] = NONE;
                        continue;
                    }
                    const uint32_t k = e - R;
                    if (k < 32u) {
                        s_rentry[w] = k;
                        e = s_rx[w][k];
                        continue;
                    }
                    // a long literal carried the chain past the region's first segment
                    s_rentry[w] = FALLBACK;
                    for (uint32_t j = 0; j < 32; ++j) {
                        const uint32_t Sj = R + SEG * j;
                        const uint32_t lj = min(Sj + SEG, cl);
                        uint32_t rec = NONE;
                        if (e >= Sj && e < lj) {
                            rec = e;
                            e = Sj + s_tbl[e];
                        }
                        s_entry[w * 32 + j] = rec;
                    }
                }
                s_carry = t0 + e;
            }
            __syncthreads();
            uint32_t ent;
            {
                const uint32_t rk = s_rentry[wid];
                if (rk < 32u) {
                    const uint16_t r = s_chain[wid * 32 * 32 + lane * 32 + rk];
                    ent = (r == 0xffff) ? NONE : (uint32_t)r;
                } else {
                    ent = (rk == FALLBACK) ? s_entry[tid] : NONE;
                }
            }

            // ---- 5. walk the segment: output bytes, tokens, validation ----
            uint32_t cnt = 0, ntok = 0;
            bool bad = false;
            if (ent != NONE) {
                for (uint32_t p = ent; p < lim;) {
                    const uint32_t c = tb[p];
                    if (p + tok_in(c) > cl) bad = true;
                    cnt += tok_out(c);
                    ++ntok;
                    p += tok_in(c);
                }
            }
            uint64_t tot64;
            const uint64_t ex = block_excl_scan64<NT>(((uint64_t)ntok << 32) | cnt, s_scan, &tot64);
            const uint32_t total = (uint32_t)tot64, ntot = (uint32_t)(tot64 >> 32);
            carry = s_carry;
            if (__syncthreads_or(bad)) {
                err = ST_CORRUPT;
                break;
            }
            if ((uint64_t)opos + total > want) {
                err = ST_OVERRUN;
                break;
            }
            // token list; and, for every 64-byte output slice that starts
            // inside a token, that token's index (s_slice, in the exit-table
            // space, which is free now) -- unless the tile's output has more
            // slices than fit, in which case the expansion searches the list
            const uint32_t sbase = opos >> 6;
            const bool indexed = ((opos + total + 63u) >> 6) - sbase <= SLICE_CAP;
            uint16_t* s_slice = reinterpret_cast<uint16_t*>(s_tbl);
            if (ntok) {
                uint32_t j = (uint32_t)(ex >> 32), o = opos + (uint32_t)ex;
                for (uint32_t p = ent; p < lim;) {
                    const uint32_t c = tb[p];
                    s_list[j] = make_uint2(o, p | (c << 16) | ((uint32_t)tb[p + 1] << 24));
                    const uint32_t oe_tok = o + tok_out(c);
                    if (indexed)
                        for (uint32_t b = (o + 63u) & ~63u; b < oe_tok; b += 64u) s_slice[(b >> 6) - sbase] = (uint16_t)j;
                    ++j;
                    o = oe_tok;
                    p += tok_in(c);
                }
            }
            __syncthreads();

            // ---- 6. expansion: 64-byte slices of [opos, opos+total) ----
            const uint32_t ob = opos, oe = opos + total;
            for (uint32_t s0 = (ob & ~63u) + 64u * tid; s0 < oe; s0 += 64u * NT) {
                const uint32_t lo = max(s0, ob), hi = min(s0 + 64u, oe);
                if (lo >= hi) continue;
                // last token whose output starts at or before lo
                uint32_t a = 0;
                if (indexed) {
                    if (lo > ob) a = s_slice[(lo >> 6) - sbase];  // lo is a slice start here
                } else {
#pragma unroll
                    for (uint32_t step = MAXTOK / 2; step; step >>= 1) {
                        const uint32_t cand = a + step;
                        if (cand < ntot && s_list[cand].x <= lo) a = cand;
                    }
                }
                uint32_t ks = s_list[a].x, info = s_list[a].y;
                uint32_t ke = ks + tok_out((info >> 16) & 0xffu);
                for (uint32_t v0 = lo & ~15u; v0 < hi; v0 += 16) {
                    const uint32_t x0 = max(v0, lo), x1 = min(v0 + 16, hi);
                    uint64_t acc0 = 0, acc1 = 0;
                    uint32_t x = x0;
                    for (;;) {
                        if (ke <= x) {  // the previous piece ended exactly at this vector's start
                            ++a;
                            ks = ke;
                            info = s_list[a].y;
                            ke = ks + tok_out((info >> 16) & 0xffu);
                        }
                        const uint32_t c = (info >> 16) & 0xffu;
                        uint64_t w0, w1;
                        if (c <= 127u) {
                            w0 = w1 = 0x0101010101010101ull * (info >> 24);
                        } else {
                            // literal byte at output position y sits at tb[pos + 1 + y - ks]
                            lds16_unaligned(tb + (int32_t)((info & 0xffffu) + 1u + v0 - ks), w0, w1);
                        }
                        // keep bytes below x, take bytes from x on
                        const uint32_t b8 = (x - v0) * 8u;
                        const uint64_t m0 = b8 >= 64u ? ~0ull : ((1ull << b8) - 1ull);
                        const uint64_t m1 = b8 <= 64u ? 0ull : ((1ull << (b8 - 64u)) - 1ull);
                        acc0 = (acc0 & m0) | (w0 & ~m0);
                        acc1 = (acc1 & m1) | (w1 & ~m1);
                        x = min(ke, x1);
                        if (x >= x1) break;
                        ++a;
                        ks = ke;
                        info = s_list[a].y;
                        ke = ks + tok_out((info >> 16) & 0xffu);
                    }
                    if (aligned16 && x0 == v0 && x1 == v0 + 16) {
                        *reinterpret_cast<uint4*>(dst + v0) =
                            make_uint4((uint32_t)acc0, (uint32_t)(acc0 >> 32), (uint32_t)acc1, (uint32_t)(acc1 >> 32));
                    } else {  // a vector shared with the neighbouring tile, or unaligned output
                        for (uint32_t y = x0; y < x1; ++y) {
                            const uint32_t b = y - v0;
                            dst[y] = (uint8_t)((b < 8 ? acc0 >> (8 * b) : acc1 >> (8 * (b - 8))) & 0xffu);
                        }
                    }
                }
            }
            opos += total;
            __syncthreads();  // tile, tables and list are reused by the next tile
        }

        if (err == ST_OK && (opos != want || carry != clen)) err = ST_CORRUPT;
        if (tid == 0) put_status(status, chunk, err);
        __syncthreads();
    }
}

}  // namespace brle
}  // namespace gd

extern "C" gd_status_t gd_brle_decode(const uint8_t* d_data, const uint64_t* d_ptr, uint32_t n_chunks,
                                      uint64_t chunk_size, uint8_t* d_out, uint64_t out_n_bytes,
                                      uint32_t* d_status, gd_stream_t stream) {
    if (n_chunks == 0) return GD_OK;
    if (!d_data || !d_ptr || !d_out || chunk_size == 0 || chunk_size > 0x7fffffffull) return GD_ERR_INVALID_ARG;
    if (out_n_bytes > chunk_size * (uint64_t)n_chunks || out_n_bytes <= chunk_size * (uint64_t)(n_chunks - 1))
        return GD_ERR_INVALID_ARG;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    uint32_t grid = n_chunks;
    const int bps = gd_tune_get(GD_TUNE_BRLE_BLOCKS_PER_SM);
    const uint32_t cap = (uint32_t)sms * (bps > 0 ? (uint32_t)bps : 8u);
    if (grid > cap) grid = cap;
    constexpr uint32_t smem = gd::brle::SMEM;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(gd::brle::decode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        attr = true;
    }
    gd::brle::decode_kernel<<<grid, gd::brle::NT, smem, (cudaStream_t)stream>>>(d_data, d_ptr, n_chunks, chunk_size,
                                                                                d_out, out_n_bytes, d_status);
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}
