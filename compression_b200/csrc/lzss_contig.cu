// lzss_contig.cu -- LZSS contiguous-container decoder for sm_100a.
//
// Container (lzss::compress_gpu / decompress_gpu_base, include/lzss/lzss.h:
// 1060-1188): chunk c's token stream is data[end[c-1] .. end[c]) and decodes
// to out[c*chunk_size ..].  Grammar (lzss::decompress_func, lzss.h:234-305):
// a flag byte, then up to 8 tokens (LSB first) while compressed bytes remain;
// bit 1 = one literal byte, bit 0 = a 2-byte little-endian v with length
// (v & 31) + 3 and offset v >> 5 back in the chunk's own output.
//
// The reference decodes one chunk per thread.  Here one warp decodes a chunk,
// 4 flag groups (up to 32 tokens) per round:
//   * lane 0 walks the round's flag bytes (a group's byte length is
//     17 - popcount(flags) when full), then lane 8g+i decodes token i of
//     group g; a warp scan of token lengths places every token;
//   * each lane then produces output bytes of the round: a literal byte
//     directly, a match byte by following the back-reference chain (inside
//     the round) until it reaches a literal of the round or a byte of an
//     earlier round, read from a 4 KiB shared-memory ring of recent output;
//   * bytes go to the ring and, coalesced, to global memory.
#include "gd_common.cuh"

namespace gd {
namespace lzssc {

constexpr int WPB = 4;            // warps (chunks in flight) per block
constexpr uint32_t RING = 4096;   // >= 2047 bytes of history + a round's output (<= 32 * 34)

struct WarpSmem {
    uint8_t ring[RING];
    uint32_t tstart[33];  // round-relative output start of token k; [32] = the round's output
    uint32_t tinfo[32];   // literal: 0x80000000 | byte; match: offset << 8 | length
    uint32_t gstart[4], ghead[4], gcnt[4];
    uint32_t next_ip, bad;
};

__global__ void __launch_bounds__(WPB * 32) decode_kernel(const uint8_t* __restrict__ data,
                                                         const uint64_t* __restrict__ ends, uint32_t n_chunks,
                                                         uint64_t chunk_size, uint8_t* __restrict__ out,
                                                         uint64_t out_n, uint32_t* __restrict__ status) {
    __shared__ WarpSmem S_[WPB];
    const uint32_t lane = lane_id(), wid = threadIdx.x >> 5;
    WarpSmem& S = S_[wid];
    for (uint32_t c = blockIdx.x * WPB + wid; c < n_chunks; c += gridDim.x * WPB) {
        const uint64_t beg = c ? ends[c - 1] : 0, end = ends[c];
        const uint64_t obase = (uint64_t)c * chunk_size;
        uint32_t err = ST_OK;
        if (end < beg || end - beg > 0x7fffffffull || obase >= out_n) err = ST_CORRUPT;
        const uint32_t clen = err ? 0u : (uint32_t)(end - beg);
        const uint32_t want = err ? 0u : (uint32_t)(out_n - obase < chunk_size ? out_n - obase : chunk_size);
        const uint8_t* src = data + beg;
        uint8_t* dst = out + obase;
        uint32_t ip = 0, op = 0;
        while (err == ST_OK && ip < clen) {
            // ---- flag groups of this round (lane 0) ----
            if (lane == 0) {
                uint32_t p = ip;
                for (uint32_t g = 0; g < 4; ++g) {
                    uint32_t h = 0, cnt = 0;
                    if (p < clen) {
                        h = src[p];
                        // token i starts at p + 1 + 2i - (literals before it); it exists
                        // while compressed bytes remain before it
                        while (cnt < 8 && p + 1 + 2 * cnt - __popc(h & ((1u << cnt) - 1u)) < clen) ++cnt;
                        S.gstart[g] = p;
                        p = p + 1 + 2 * cnt - __popc(h & ((1u << cnt) - 1u));
                    }
                    S.ghead[g] = h;
                    S.gcnt[g] = cnt;
                    if (cnt < 8) {  // the chunk's stream ends in this group
                        for (uint32_t g2 = g + 1; g2 < 4; ++g2) S.gcnt[g2] = 0;
                        break;
                    }
                }
                S.next_ip = p;
            }
            __syncwarp();
            // ---- token of this lane ----
            const uint32_t g = lane >> 3, i = lane & 7u;
            const uint32_t h = S.ghead[g];
            const bool has = i < S.gcnt[g];
            uint32_t len = 0, info = 0;
            bool bad = false;
            if (has) {
                const uint32_t pos = S.gstart[g] + 1 + 2 * i - __popc(h & ((1u << i) - 1u));
                if ((h >> i) & 1u) {
                    len = 1;
                    info = 0x80000000u | src[pos];
                } else if (pos + 2 > clen) {
                    bad = true;
                } else {
                    const uint32_t v = (uint32_t)src[pos] | ((uint32_t)src[pos + 1] << 8);
                    len = (v & 31u) + 3u;
                    info = ((v >> 5) << 8) | len;
                }
            }
            const uint32_t inc = warp_incl_scan(len);
            const uint32_t ostart = inc - len, T = __shfl_sync(GD_FULL_MASK, inc, 31);
            if (has && !bad && !(info >> 31)) {
                const uint32_t off = info >> 8;
                if (off == 0 || off > op + ostart) bad = true;  // before the chunk's first byte
            }
            if (__any_sync(GD_FULL_MASK, bad)) {
                err = ST_CORRUPT;
                break;
            }
            if ((uint64_t)op + T > want) {
                err = ST_OVERRUN;
                break;
            }
            S.tstart[lane] = has ? ostart : T;
            S.tinfo[lane] = info;
            if (lane == 0) S.tstart[32] = T;
            __syncwarp();
            // ---- output bytes of the round ----
            for (uint32_t b = lane; b < T; b += 32) {
                uint32_t r = b;  // round-relative position whose value is wanted
                uint32_t val;
                for (;;) {
                    uint32_t k = 0;  // last token starting at or before r
#pragma unroll
                    for (uint32_t step = 16; step; step >>= 1)
                        if (S.tstart[k + step] <= r) k += step;
                    const uint32_t tk = S.tinfo[k];
                    if (tk >> 31) {
                        val = tk & 0xffu;
                        break;
                    }
                    const uint32_t q = op + r - (tk >> 8);  // absolute source position
                    if (q < op) {
                        val = S.ring[q & (RING - 1)];
                        break;
                    }
                    r = q - op;
                }
                S.ring[(op + b) & (RING - 1)] = (uint8_t)val;
                dst[op + b] = (uint8_t)val;
            }
            __syncwarp();
            op += T;
            ip = S.next_ip;
            __syncwarp();
        }
        if (err == ST_OK && (ip != clen || op != want)) err = ST_CORRUPT;
        if (lane == 0) put_status(status, c, err);
        __syncwarp();
    }
}

}  // namespace lzssc
}  // namespace gd

extern "C" gd_status_t gd_lzss_contig_decode(const uint8_t* d_data, const uint64_t* d_ends, uint32_t n_chunks,
                                             uint64_t chunk_size, uint8_t* d_out, uint64_t out_n_bytes,
                                             uint32_t* d_status, gd_stream_t stream) {
    if (n_chunks == 0) return GD_OK;
    if (!d_data || !d_ends || !d_out || chunk_size == 0 || chunk_size > 0xffffffffull) return GD_ERR_INVALID_ARG;
    if (out_n_bytes > chunk_size * (uint64_t)n_chunks || out_n_bytes <= chunk_size * (uint64_t)(n_chunks - 1))
        return GD_ERR_INVALID_ARG;
    using namespace gd::lzssc;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    uint32_t grid = (n_chunks + WPB - 1) / WPB;
    const uint32_t cap = (uint32_t)sms * 16;
    if (grid > cap) grid = cap;
    decode_kernel<<<grid, WPB * 32, 0, (cudaStream_t)stream>>>(d_data, d_ends, n_chunks, chunk_size, d_out,
                                                              out_n_bytes, d_status);
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}
