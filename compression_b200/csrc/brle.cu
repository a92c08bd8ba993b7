// brle.cu -- byte-RLE (brle.h container) decoder for sm_100a.
//
// Format (restated from brle::decode, include/brle/brle.h:76-97): a chunk is
// a sequence of tokens; control byte c > 127 is followed by c-127 literal
// bytes, c <= 127 by one byte repeated c+3 times.  Chunk c's tokens occupy
// data[ptr[c] .. ptr[c+1]) and expand to out[c*chunk_size ..].
//
// The reference decodes one chunk per thread (1024 threads on the whole GPU
// for a 256 MiB column).  Here one 256-thread block decodes a chunk:
//   1. An 8 KiB tile of compressed bytes is staged in shared memory.
//   2. Token starts: every thread walks the token chain speculatively from
//      the start of its 32-byte segment, recording the token starts it meets
//      (a bit mask) and where the chain leaves the segment.  One thread then
//      joins the segments: when the true chain enters a segment at a recorded
//      start, the speculative walk is already correct from there on; only
//      segments entered elsewhere are re-walked.
//   3. A block scan of per-thread output sizes places every token.
//   4. Tokens are expanded into a 16 KiB shared-memory window (runs as 32-bit
//      fills) that is written to HBM with coalesced 16-byte stores.
// Every read is bounded by the chunk's compressed length and every write by
// its output size; a malformed chunk gets GD_ERR_CORRUPT / GD_ERR_OVERRUN.
#include "gd_common.cuh"

namespace gd {
namespace brle {

constexpr int NT = 256;
constexpr int SEG = 32;
constexpr int TILE = NT * SEG;  // compressed bytes per tile
constexpr int HALO = 160;       // a token starting in the tile reads <= 129 more bytes
constexpr int OUTW = 16384;     // output window staged in shared memory

__device__ __forceinline__ uint32_t tok_in(uint32_t c) { return c > 127u ? c - 126u : 2u; }
__device__ __forceinline__ uint32_t tok_out(uint32_t c) { return c > 127u ? c - 127u : c + 3u; }

// Fill window bytes [lo, hi) (window-relative) with value v.
__device__ __forceinline__ void win_fill(uint8_t* win, uint32_t lo, uint32_t hi, uint8_t v) {
    uint32_t rep = 0x01010101u * v;
    while (lo < hi && (lo & 3u)) win[lo++] = v;
    while (lo + 4 <= hi) {
        *reinterpret_cast<uint32_t*>(win + lo) = rep;
        lo += 4;
    }
    while (lo < hi) win[lo++] = v;
}

__global__ void __launch_bounds__(NT) decode_kernel(const uint8_t* __restrict__ data,
                                                    const uint64_t* __restrict__ ptr, uint32_t n_chunks,
                                                    uint64_t chunk_size, uint8_t* __restrict__ out,
                                                    uint64_t out_n, uint32_t* __restrict__ status) {
    __shared__ __align__(16) uint8_t s_tile[TILE + HALO + 16];
    __shared__ __align__(16) uint8_t s_win[OUTW];
    __shared__ uint32_t s_mask[NT];
    __shared__ uint32_t s_exit[NT];
    __shared__ uint32_t s_scan[NT / 32 + 1];
    __shared__ uint32_t s_carry;

    const uint32_t tid = threadIdx.x;
    for (uint32_t chunk = blockIdx.x; chunk < n_chunks; chunk += gridDim.x) {
        const uint64_t beg = ptr[chunk], end = ptr[chunk + 1];
        const uint64_t obase = (uint64_t)chunk * chunk_size;
        uint32_t err = ST_OK;
        if (end < beg || end - beg > 0x7fffffffull || obase >= out_n) err = ST_CORRUPT;
        const uint32_t clen = err ? 0u : (uint32_t)(end - beg);
        const uint64_t want64 = err ? 0 : (out_n - obase < chunk_size ? out_n - obase : chunk_size);
        const uint32_t want = (uint32_t)want64;
        const uint8_t* src = data + beg;
        uint8_t* dst = out + obase;
        const bool aligned = ((reinterpret_cast<uintptr_t>(dst) & 15u) == 0);

        uint32_t carry = 0;  // chunk-relative position of the next token start
        uint32_t opos = 0;   // output bytes placed so far
        uint32_t W = 0;      // chunk-relative start of the staging window

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

            // ---- 2a. speculative walk of this thread's segment ----
            const uint32_t S = t0 + SEG * tid;
            {
                uint32_t m = 0, p = S;
                const uint32_t lim = min(S + SEG, clen);
                while (p < lim) {
                    m |= 1u << (p - S);
                    p += tok_in(tb[p - t0]);
                }
                s_mask[tid] = m;
                s_exit[tid] = p;
            }
            __syncthreads();

            // ---- 2b. join segments along the true chain ----
            if (tid == 0) {
                uint32_t e = carry;
                for (uint32_t t = 0; t < (uint32_t)NT; ++t) {
                    const uint32_t St = t0 + SEG * t;
                    if (St >= clen) break;  // masks beyond the data are already 0
                    if (e >= St + SEG) {
                        s_mask[t] = 0;
                        continue;
                    }
                    const uint32_t k = e - St;
                    const uint32_t m = s_mask[t];
                    if ((m >> k) & 1u) {
                        s_mask[t] = m & (~0u << k);
                        e = s_exit[t];
                    } else {
                        uint32_t mm = 0, p = e;
                        const uint32_t lim = min(St + SEG, clen);
                        while (p < lim) {
                            mm |= 1u << (p - St);
                            p += tok_in(tb[p - t0]);
                        }
                        s_mask[t] = mm;
                        e = p;
                    }
                }
                s_carry = e;
            }
            __syncthreads();

            // ---- 3. per-thread output size + validation, block scan ----
            const uint32_t mask = s_mask[tid];
            uint32_t cnt = 0;
            bool bad = false;
            {
                uint32_t m = mask;
                while (m) {
                    const uint32_t b = __ffs(m) - 1;
                    m &= m - 1;
                    const uint32_t p = S + b;
                    const uint32_t c = tb[p - t0];
                    if (p + tok_in(c) > clen) bad = true;
                    cnt += tok_out(c);
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

            // ---- 4. expand through the staging window ----
            uint32_t m_rem = mask;
            uint32_t cur = opos + excl;  // output offset of the first remaining token
            const uint32_t tile_end = opos + total;
            for (;;) {
                const uint32_t whi = W + OUTW;
                while (m_rem) {
                    const uint32_t b = __ffs(m_rem) - 1;
                    const uint32_t p = S + b;
                    const uint32_t c = tb[p - t0];
                    const uint32_t len = tok_out(c);
                    if (cur >= whi) break;
                    const uint32_t lo = max(cur, W), hi = min(cur + len, whi);
                    if (c <= 127u) {
                        win_fill(s_win, lo - W, hi - W, tb[p - t0 + 1]);
                    } else {
                        const uint8_t* lit = tb + (p - t0 + 1) + (lo - cur);
                        for (uint32_t x = lo; x < hi; ++x) s_win[x - W] = *lit++;
                    }
                    if (cur + len > whi) break;  // continues in the next window
                    cur += len;
                    m_rem &= m_rem - 1;
                }
                __syncthreads();
                if (tile_end < whi) break;  // window not complete yet
                // flush the full window [W, W+OUTW)
                if (aligned) {
                    uint4* d4 = reinterpret_cast<uint4*>(dst + W);
                    const uint4* s4 = reinterpret_cast<const uint4*>(s_win);
                    for (uint32_t i = tid; i < OUTW / 16; i += NT) d4[i] = s4[i];
                } else {
                    for (uint32_t i = tid; i < OUTW; i += NT) dst[W + i] = s_win[i];
                }
                __syncthreads();
                W += OUTW;
                if (tile_end == W) break;
            }
            opos = tile_end;
        }

        if (err == ST_OK && opos != want) err = ST_CORRUPT;
        if (err == ST_OK && opos > W) {
            // flush the final partial window [W, want)
            const uint32_t n = want - W;
            if (aligned) {
                uint4* d4 = reinterpret_cast<uint4*>(dst + W);
                const uint4* s4 = reinterpret_cast<const uint4*>(s_win);
                for (uint32_t i = tid; i < n / 16; i += NT) d4[i] = s4[i];
                for (uint32_t i = (n & ~15u) + tid; i < n; i += NT) dst[W + i] = s_win[i];
            } else {
                for (uint32_t i = tid; i < n; i += NT) dst[W + i] = s_win[i];
            }
        }
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
    gd::brle::decode_kernel<<<grid, gd::brle::NT, 0, (cudaStream_t)stream>>>(d_data, d_ptr, n_chunks, chunk_size,
                                                                             d_out, out_n_bytes, d_status);
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}
