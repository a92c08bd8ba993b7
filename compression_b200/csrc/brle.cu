// brle.cu -- byte-RLE (brle.h container) decoder for sm_100a.
//
// Format (restated from brle::decode, include/brle/brle.h:76-97): a chunk is
// a sequence of tokens; control byte c > 127 is followed by c-127 literal
// bytes, c <= 127 by one byte repeated c+3 times.  Chunk c's tokens occupy
// data[ptr[c] .. ptr[c+1]) and expand to out[c*chunk_size ..].
//
// The reference decodes one chunk per thread (1024 threads on the whole GPU
// for a 256 MiB column).  Here one 256-thread block decodes a chunk, 16 KiB
// of compressed bytes (a tile) at a time:
//   1. The tile (8 KiB) is staged in shared memory with 16-byte loads.
//   2. Token starts form a chain (each token is 2..129 bytes).  Thread t owns
//      a 32-byte segment and computes, by one backward pass over its bytes,
//      where the chain leaves the segment for every possible entry offset
//      (a 32-entry exit table).  One thread then follows the chain across
//      the 256 segments with one table lookup each; the other tables make
//      any entry O(1), so no speculation or re-walking is needed.
//   3. Each thread walks its segment from its true entry; a block scan of
//      output sizes places every token, and each warp packs its tokens into a
//      list of (output offset, tile position).
//   4. Each warp expands its output range in rounds of 32 x 64 bytes: lane l
//      takes the 64-byte slice l of the round (equal work per lane whatever
//      the token lengths), finds the token covering its first byte by binary
//      search in the list, and builds aligned 16-byte vectors in registers
//      (a vector inside one run is a single broadcast value) which it stores
//      straight to HBM.  Bytes of 16-byte words shared with a neighbouring
//      warp are stored bytewise.
// Every read is bounded by the chunk's compressed length and every write by
// its output size; a malformed chunk gets GD_ERR_CORRUPT / GD_ERR_OVERRUN.
#include "gd_common.cuh"

namespace gd {
namespace brle {

constexpr int NT = 256;
constexpr int NWARP = NT / 32;
constexpr int SEG = 32;         // compressed bytes per thread segment
constexpr int TILE = NT * SEG;  // compressed bytes per tile
constexpr int HALO = 160;       // a token starting in the tile reads <= 129 more bytes
constexpr uint32_t NONE = 0xffffffffu;
constexpr uint32_t TPW = 32 * SEG / 2;  // most tokens a warp's segments can hold
constexpr uint32_t SMEM = TILE + HALO + 16 + NT * SEG + NWARP * TPW * 6;

__device__ __forceinline__ uint32_t tok_in(uint32_t c) { return c > 127u ? c - 126u : 2u; }
__device__ __forceinline__ uint32_t tok_out(uint32_t c) { return c > 127u ? c - 127u : c + 3u; }

__global__ void __launch_bounds__(NT) decode_kernel(const uint8_t* __restrict__ data,
                                                    const uint64_t* __restrict__ ptr, uint32_t n_chunks,
                                                    uint64_t chunk_size, uint8_t* __restrict__ out,
                                                    uint64_t out_n, uint32_t* __restrict__ status) {
    extern __shared__ __align__(16) uint8_t s_dyn[];
    uint8_t* s_tile = s_dyn;                          // TILE + HALO + 16
    uint8_t* s_tbl = s_dyn + TILE + HALO + 16;        // NT x SEG exit tables, then token lists
    __shared__ uint32_t s_entry[NT];
    __shared__ uint32_t s_scan[NWARP + 1];
    __shared__ uint32_t s_carry;

    const uint32_t tid = threadIdx.x, lane = tid & 31u, wid = tid >> 5;
    // token list of this warp: output offsets and tile positions
    uint32_t* tl_out = reinterpret_cast<uint32_t*>(s_tbl + NT * SEG) + wid * TPW;
    uint16_t* tl_pos = reinterpret_cast<uint16_t*>(s_tbl + NT * SEG + NWARP * TPW * 4) + wid * TPW;
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
            // ---- 1. stage compressed bytes [t0, min(clen, t0+TILE+HALO)) ----
            // Tile byte i lives at tb[i] = s_tile[sh + i], sh = the global
            // address mod 16, so aligned 16-byte global words land on aligned
            // shared words; the ragged head and tail are copied bytewise.
            const uint32_t n_ld = min(clen - t0, (uint32_t)(TILE + HALO));
            const uint8_t* g = src + t0;
            const uint32_t sh = (uint32_t)(reinterpret_cast<uintptr_t>(g) & 15u);
            const uint8_t* tb = s_tile + sh;
            {
                uint32_t head = (16u - sh) & 15u;
                if (head > n_ld) head = n_ld;
                if (tid < head) s_tile[sh + tid] = g[tid];
                const uint32_t nv = (n_ld - head) >> 4;
                const uint4* gv = reinterpret_cast<const uint4*>(g + head);
                uint4* sv = reinterpret_cast<uint4*>(s_tile + sh + head);
                for (uint32_t i = tid; i < nv; i += NT) sv[i] = __ldg(gv + i);
                for (uint32_t i = head + 16 * nv + tid; i < n_ld; i += NT) s_tile[sh + i] = g[i];
            }
            __syncthreads();

            // ---- 2a. exit table of this thread's segment ----
            // tbl[k] = (chain exit - S) when the chain enters at S + k; an
            // exit is the first chain position >= lim (<= 64 + 129 - 1).
            const uint32_t S = t0 + SEG * tid;
            const uint32_t lim = min(S + SEG, clen);
            uint8_t* tbl = s_tbl + tid * SEG;
            if (S < clen) {
                for (int32_t p = (int32_t)lim - 1; p >= (int32_t)S; --p) {
                    const uint32_t n = (uint32_t)p + tok_in(tb[(uint32_t)p - t0]);
                    tbl[(uint32_t)p - S] = (n >= lim) ? (uint8_t)(n - S) : tbl[n - S];
                }
            }
            __syncthreads();

            // ---- 2b. follow the chain across the segments (one lookup each) ----
            if (tid == 0) {
                uint32_t e = carry;
                for (uint32_t t = 0; t < (uint32_t)NT; ++t) {
                    const uint32_t St = t0 + SEG * t;
                    if (St >= clen || e >= min(St + SEG, clen)) {
                        s_entry[t] = NONE;  // no token starts in segment t
                        continue;
                    }
                    s_entry[t] = e;
                    e = St + s_tbl[t * SEG + (e - St)];
                }
                s_carry = e;
            }
            __syncthreads();

            // ---- 3. token starts, output size, validation; scans; token list ----
            uint32_t mask = 0;
            uint32_t cnt = 0;
            bool bad = false;
            {
                const uint32_t e = s_entry[tid];
                if (e != NONE) {
                    uint32_t p = e;
                    while (p < lim) {
                        mask |= 1u << (p - S);
                        const uint32_t c = tb[p - t0];
                        if (p + tok_in(c) > clen) bad = true;
                        cnt += tok_out(c);
                        p += tok_in(c);
                    }
                }
            }
            uint32_t total;
            const uint32_t excl = block_excl_scan<NT>(cnt, s_scan, &total);
            carry = s_carry;
            if (__syncthreads_or(bad)) {
                err = ST_CORRUPT;
                break;
            }
            if ((uint64_t)opos + total > want) {
                err = ST_OVERRUN;
                break;
            }
            const uint32_t ntok = __popc(mask);
            const uint32_t tinc = warp_incl_scan(ntok);
            const uint32_t n_w = __shfl_sync(GD_FULL_MASK, tinc, 31);  // tokens of this warp
            {
                uint32_t j = tinc - ntok, o = opos + excl;
                uint32_t m = mask;
                while (m) {
                    const uint32_t tp = S + (__ffs(m) - 1) - t0;
                    tl_out[j] = o;
                    tl_pos[j] = (uint16_t)tp;
                    o += tok_out(tb[tp]);
                    ++j;
                    m &= m - 1;
                }
            }
            __syncwarp();

            // ---- 4. merge-path expansion: 64 output bytes per lane per round ----
            if (n_w) {
                const uint32_t wbeg = __shfl_sync(GD_FULL_MASK, opos + excl, 0);
                const uint32_t wend = __shfl_sync(GD_FULL_MASK, opos + excl + cnt, 31);
                for (uint32_t r = wbeg & ~15u; r < wend; r += 32 * 64) {
                    const uint32_t lo = max(r + 64 * lane, wbeg);
                    const uint32_t hi = min(r + 64 * lane + 64, wend);
                    if (lo >= hi) continue;
                    // last token whose output starts at or before lo
                    uint32_t a = 0, b = n_w;  // invariant: tl_out[a] <= lo < tl_out[b]
                    while (b - a > 1) {
                        const uint32_t m = (a + b) >> 1;
                        if (tl_out[m] <= lo) a = m;
                        else b = m;
                    }
                    uint32_t k = a;
                    uint32_t ks = tl_out[k], kp = tl_pos[k];
                    uint32_t kc = tb[kp];
                    uint32_t ke = ks + tok_out(kc);
                    for (uint32_t v0 = lo & ~15u; v0 < hi; v0 += 16) {
                        const uint32_t x0 = max(v0, lo), x1 = min(v0 + 16, hi);
                        while (ke <= x0) {  // advance to the token covering x0
                            ++k;
                            ks = ke;
                            kp = tl_pos[k];
                            kc = tb[kp];
                            ke = ks + tok_out(kc);
                        }
                        if (aligned16 && x0 == v0 && x1 == v0 + 16 && kc <= 127u && ke >= x1) {
                            const uint32_t rep = 0x01010101u * tb[kp + 1];
                            *reinterpret_cast<uint4*>(dst + v0) = make_uint4(rep, rep, rep, rep);
                            continue;
                        }
                        uint32_t w[4] = {0, 0, 0, 0};
                        uint32_t x = x0;
                        for (;;) {
                            const uint32_t n = min(ke, x1) - x;
                            if (kc <= 127u) {
                                const uint32_t rep = 0x01010101u * tb[kp + 1];
#pragma unroll
                                for (uint32_t q = 0; q < 4; ++q) {
                                    const uint32_t ql = v0 + 4 * q;
                                    const uint32_t a0 = max(x, ql), a1 = min(x + n, ql + 4);
                                    if (a0 < a1) {
                                        const uint32_t nb = a1 - a0;
                                        const uint32_t msk = (nb == 4 ? 0xffffffffu : ((1u << (8 * nb)) - 1u)) << (8 * (a0 - ql));
                                        w[q] = (w[q] & ~msk) | (rep & msk);
                                    }
                                }
                            } else {
                                const uint8_t* lit = tb + kp + 1 + (x - ks);
                                for (uint32_t i = 0; i < n; ++i) {
                                    const uint32_t bo = x - v0 + i;
                                    w[bo >> 2] |= (uint32_t)lit[i] << (8 * (bo & 3u));
                                }
                            }
                            x += n;
                            if (x >= x1) break;
                            ++k;
                            ks = ke;
                            kp = tl_pos[k];
                            kc = tb[kp];
                            ke = ks + tok_out(kc);
                        }
                        if (aligned16 && x0 == v0 && x1 == v0 + 16) {
                            *reinterpret_cast<uint4*>(dst + v0) = make_uint4(w[0], w[1], w[2], w[3]);
                        } else {  // partial word (shared with a neighbouring warp) or unaligned output
                            for (uint32_t y = x0; y < x1; ++y) dst[y] = (uint8_t)(w[(y - v0) >> 2] >> (8 * ((y - v0) & 3u)));
                        }
                    }
                }
            }
            opos += total;
            __syncthreads();  // tile, tables and lists are reused by the next tile
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
    const uint32_t cap = (uint32_t)sms * 8;
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
